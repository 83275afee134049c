"""GPU parity at the sizes of the benchmark configurations, against the
oracle (not the GPU's own FP64 solve):

  * the 64 x 64 quad4 plate of the plain configuration (8,450 dofs, E = 70e3,
    nu = 0.3, left edge clamped, traction 1.0 on the right edge), FP64
    Jacobi-PCG under the reference's stop rule sqrt(r.r/x.x) < 1e-10
    (sparse.cpp:223): pattern bit-exact, FP64 K within 1e-12 of the row's
    largest entry, the oracle's iteration count within 2 %, and the solution
    the oracle's;
  * a cube of the precision configuration's generator (lognormal E, random
    nu, z = 0 clamped, pressure on z = 1) at 50^3 (397,953 dofs; its FP32
    node-block matrix, 138 MB, is larger than L2): FP32 K within 1e-5 of the
    row's largest entry (entries that are small by cancellation carry the
    rounding of the row's large terms, so the bound is scaled by the row),
    and the mixed-precision solution within 1e-8 (relative L2) of the
    oracle's FP64 solution converged to ||r||/||b|| <= 1e-13.
"""
import numpy as np
import pytest

from betanoox_b200 import Solver, _abi, opts
from betanoox_b200 import workloads as W

pytestmark = pytest.mark.gpu


def row_scaled_err(rp, ref, got):
    """max over rows of max|got - ref| / max|ref| (rows of 0-based CSR rp)."""
    rp = np.asarray(rp, np.int64)
    d = np.abs(np.asarray(got) - np.asarray(ref))
    a = np.abs(np.asarray(ref))
    nz = np.diff(rp) > 0
    starts = rp[:-1][nz]
    dm = np.maximum.reduceat(d, starts)
    am = np.maximum.reduceat(a, starts)
    am[am == 0] = 1.0
    return float((dm / am).max())


def _oracle(oracle, m, threaded=False):
    s = oracle.System(m)
    assert s.set_bc(m.restrained, m.prescribed, m.load) == 0
    s.build_pattern()
    assert (s.assemble_threaded(m.params, m.order) if threaded else s.assemble(m.params, m.order)) == 0
    return s


def test_plate64_fp64_reference_rule(oracle):
    m = W.plate_quad4(64)
    assert m.ndof == 8450
    s = _oracle(oracle, m)
    rp, col, val = s.export_lower()
    g = Solver()
    g.load_model(m)
    assert g.build_pattern() == len(col)
    rp2, col2 = g.pattern_lower()
    np.testing.assert_array_equal(rp, rp2)
    np.testing.assert_array_equal(col, col2)
    g.assemble(_abi.FP64)
    v2, _ = g.lower_values(_abi.FP64)
    assert row_scaled_err(rp, val, v2) <= 1e-12
    rc, u_ref, st_ref = s.solve(eps=1e-10, maxit=100000)
    assert rc == 0
    rc, st = g.solve(opts(mode=_abi.MODE_FP64, stop_rule=_abi.STOP_REF, tol=1e-10, maxit=100000))
    assert rc == _abi.OK
    u = g.download()
    assert abs(st.iterations - st_ref.iterations) <= max(2, 0.02 * st_ref.iterations), (st.iterations, st_ref.iterations)
    # same algorithm, same stop rule: the same iterate up to rounding
    assert np.linalg.norm(u - u_ref) <= 1e-9 * np.linalg.norm(u_ref)
    # and mixed precision reaches the oracle's tight solution
    rc, u_t, _ = s.solve(eps=1e-14, maxit=200000)
    assert rc in (0, oracle.ERR_MAXIT)
    g.assemble(_abi.FP32)
    rc, st = g.solve(opts(mode=_abi.MODE_MPIR, tol=1e-12))
    assert rc == _abi.OK
    assert np.linalg.norm(g.download() - u_t) <= 1e-8 * np.linalg.norm(u_t)


@pytest.fixture(scope="module")
def cube50(oracle):
    m = W.cube_hex8(50)
    s = _oracle(oracle, m, threaded=True)
    rp, col, val = s.export_lower()
    csr = s.csr()
    b = s.rhs()
    x0 = np.where(np.asarray(m.restrained, bool), m.prescribed, 0.0)
    rc, u_t, st, _ = csr.pcg(b, 1e-13, maxit=200000, rule=oracle.Csr.RULE_RB, x0=x0)
    assert rc == 0
    return m, rp, col, val, u_t


def test_cube50_fp32_assembly(cube50):
    m, rp, col, val, _ = cube50
    g = Solver()
    g.load_model(m)
    g.build_pattern()
    rp2, col2 = g.pattern_lower()
    np.testing.assert_array_equal(rp, rp2)
    np.testing.assert_array_equal(col, col2)
    g.assemble(_abi.FP32)
    v2, _ = g.lower_values(_abi.FP32)
    assert row_scaled_err(rp, val, v2) <= 1e-5
    g.assemble(_abi.FP64)
    v3, _ = g.lower_values(_abi.FP64)
    assert row_scaled_err(rp, val, v3) <= 1e-12


@pytest.mark.parametrize("mode", [_abi.MODE_MPIR, _abi.MODE_FP64])
def test_cube50_solution_within_1e8_of_the_oracle(cube50, mode):
    m, _, _, _, u_t = cube50
    g = Solver()
    g.load_model(m)
    g.build_pattern()
    g.assemble(_abi.FP32 if mode == _abi.MODE_MPIR else _abi.FP64)
    rc, st = g.solve(opts(mode=mode, precond=_abi.PRECOND_BLOCK_JACOBI if mode == _abi.MODE_MPIR
                          else _abi.PRECOND_JACOBI, stop_rule=_abi.STOP_RB, tol=1e-10))
    assert rc == _abi.OK
    u = g.download()
    err = np.linalg.norm(u - u_t) / np.linalg.norm(u_t)
    assert err <= 1e-8, (err, st.as_dict())
