"""The geometric-nonlinear Newton loop on the GPU (BasicModel::iterate,
BasicModel.cpp:1244-1381, with ElasticityElement3D in its
GEOMETRIC_NONLINEAR form) against the oracle's restatement, which is pinned
to the reference's own element code (tests/test_oracle_pins.py):

  * the nonlinear internal force at a large displacement within 1e-12;
  * the tangent assembled at that displacement: pattern bit-exact, FP64
    within 1e-12 and FP32 within 1e-5 of the row's largest entry;
  * a cantilever loaded into large rotation (tip deflection about a fifth of
    its length): the FP64 loop takes the oracle's Newton steps (the same
    count, each iteration's max |residual| within 1e-6 while it is large)
    and ends within 1e-8 of the oracle's displacement; the mixed loop (FP32
    tangent and inner PCG, FP64 residual) reaches the same displacement.
"""
import numpy as np
import pytest

from betanoox_b200 import Solver, _abi, opts
from betanoox_b200 import workloads as W

pytestmark = pytest.mark.gpu

LOAD = 12.0


def _row_scaled(rp, ref, got):
    rp = np.asarray(rp, np.int64)
    d = np.abs(np.asarray(got) - np.asarray(ref))
    a = np.abs(np.asarray(ref))
    starts = rp[:-1][np.diff(rp) > 0]
    am = np.maximum.reduceat(a, starts)
    am[am == 0] = 1.0
    return float((np.maximum.reduceat(d, starts) / am).max())


@pytest.fixture(scope="module")
def beam(oracle):
    m = W.cantilever_hex8(nx=16, ny=2, nz=2, load=LOAD)
    s = oracle.System(m)
    s.set_bc(m.restrained, m.prescribed, m.load)
    s.build_pattern()
    rc, u, hist, its, lin = s.newton(m.params, m.order, np.zeros(m.ndof), max_residual=1e-10, max_newton=60,
                                     eps=1e-12)
    assert rc == 0
    return m, s, u, hist


def test_internal_force_and_tangent(oracle, beam):
    m, s, u_ref, _ = beam
    g = Solver()
    g.load_model(m)
    g.build_pattern()
    f = g.internal_force_nonlinear(u_ref)
    f_ref = oracle.internal_force_gnl_hex8(m, m.params, m.order, u_ref)
    assert np.linalg.norm(f - f_ref) <= 1e-12 * np.linalg.norm(f_ref)
    s.assemble_gnl(m.params, m.order, u_ref)
    rp, col, val = s.export_lower()
    g.set_solution(u_ref)
    rp2, col2 = g.pattern_lower()
    np.testing.assert_array_equal(rp, rp2)
    np.testing.assert_array_equal(col, col2)
    g.assemble(_abi.FP64, _abi.ASM_TANGENT)
    v64, _ = g.lower_values(_abi.FP64)
    assert _row_scaled(rp, val, v64) <= 1e-12
    g.assemble(_abi.FP32, _abi.ASM_TANGENT)
    v32, _ = g.lower_values(_abi.FP32)
    assert _row_scaled(rp, val, v32) <= 1e-5
    # a tangent is not a static stiffness: the linear solve refuses it
    rc, _ = g.solve(opts(mode=_abi.MODE_MPIR), raise_on_error=False)
    assert rc == _abi.ERR_STATE


def test_fp64_newton_takes_the_oracles_steps(beam):
    m, _, u_ref, hist_ref = beam
    g = Solver()
    g.load_model(m)
    g.build_pattern()
    rc, st, hist = g.newton(opts(mode=_abi.MODE_FP64, stop_rule=_abi.STOP_REF, tol=1e-12, maxit=100000),
                            max_residual=1e-10, max_newton=60)
    assert rc == _abi.OK, st.as_dict()
    assert st.iterations == len(hist_ref) - 1
    big = hist_ref > 1e-4
    np.testing.assert_allclose(hist[big], hist_ref[big], rtol=1e-6)
    u = g.download()
    assert np.linalg.norm(u - u_ref) <= 1e-8 * np.linalg.norm(u_ref)
    assert st.max_residual < 1e-10
    tip = np.isclose(m.xyz[:, 0], m.meta["length"])
    assert -u[3 * np.nonzero(tip)[0] + 2].mean() > 0.15 * m.meta["length"]  # large rotation


def test_mixed_newton_reaches_the_oracles_solution(beam):
    m, _, u_ref, hist_ref = beam
    g = Solver()
    g.load_model(m)
    g.build_pattern()
    rc, st, hist = g.newton(opts(mode=_abi.MODE_MPIR, precond=_abi.PRECOND_BLOCK_JACOBI, inner_tol=1e-4,
                                 maxit=100000), max_residual=1e-10, max_newton=60)
    assert rc == _abi.OK, st.as_dict()
    assert st.max_residual < 1e-10 and hist[-1] < 1e-10
    u = g.download()
    assert np.linalg.norm(u - u_ref) <= 1e-8 * np.linalg.norm(u_ref)
    assert st.iterations <= 2 * (len(hist_ref) - 1) + 4
