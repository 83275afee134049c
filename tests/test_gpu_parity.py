"""GPU parity: the sm_100a path through the C ABI against the oracle.

Tolerances (stated by the build's accuracy contract):
  * integer structure (lower-triangle pattern): bit-exact;
  * assembled K in FP64: |K_gpu - K_ref| <= 1e-12 * max|K_ref| of the row;
  * assembled K in FP32: |K_gpu - K_ref| <= 1e-5  * max|K_ref| of the row;
  * solutions: relative L2 error <= 1e-8 against a tightly converged FP64
    oracle solution (mixed precision after refinement, and plain FP64).
"""
import ctypes as C

import numpy as np
import pytest

from betanoox_b200 import Solver, _abi, opts
from betanoox_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _oracle_system(oracle, m, assemble=True):
    s = oracle.System(m)
    assert s.set_bc(m.restrained, m.prescribed, m.load) == 0
    s.build_pattern()
    if assemble:
        assert s.assemble(m.params, m.order) == 0
    return s


def _row_scaled_err(rp, ref, got):
    worst = 0.0
    for i in range(len(rp) - 1):
        a, b = rp[i], rp[i + 1]
        scale = np.abs(ref[a:b]).max()
        if scale == 0:
            scale = 1.0
        worst = max(worst, np.abs(ref[a:b] - got[a:b]).max() / scale)
    return worst


MODELS = {
    "quad4": lambda: W.plate_quad4(12),
    "hex8": lambda: W.cube_hex8(6, seed=11),
    "heat": lambda: W.heat_slab(8, 7, 5, order=3),
    "rve": lambda: W.rve_hex8(7, 5),
    "heat2d": lambda: W.heat_plate(12, 9, heat=2.0),
}


@pytest.mark.parametrize("name", list(MODELS))
def test_pattern_and_fp64_assembly(oracle, name):
    m = MODELS[name]()
    s = _oracle_system(oracle, m)
    rp, col, val = s.export_lower()
    pl = s.pseudo_load()
    g = Solver()
    g.load_model(m)
    assert g.build_pattern() == len(col)
    rp2, col2 = g.pattern_lower()
    np.testing.assert_array_equal(rp, rp2)
    np.testing.assert_array_equal(col, col2)
    g.assemble(_abi.FP64)
    v2, pl2 = g.lower_values(_abi.FP64)
    assert _row_scaled_err(rp, val, v2) <= 1e-12
    assert np.abs(pl - pl2).max() <= 1e-12 * max(1.0, np.abs(pl).max())


@pytest.mark.parametrize("name", list(MODELS))
def test_fp32_assembly(oracle, name):
    m = MODELS[name]()
    s = _oracle_system(oracle, m)
    rp, col, val = s.export_lower()
    g = Solver()
    g.load_model(m)
    g.build_pattern()
    g.assemble(_abi.FP32)
    v2, _ = g.lower_values(_abi.FP32)
    assert _row_scaled_err(rp, val, v2) <= 1e-5


def test_assembly_is_deterministic():
    m = W.cube_hex8(5, seed=4)
    out = []
    for _ in range(2):
        g = Solver()
        g.load_model(m)
        g.build_pattern()
        g.assemble(_abi.FP64)
        out.append(g.lower_values(_abi.FP64)[0])
    np.testing.assert_array_equal(out[0], out[1])


@pytest.mark.parametrize("name", ["quad4", "hex8", "heat", "heat2d"])
def test_matvec(oracle, name):
    m = MODELS[name]()
    s = _oracle_system(oracle, m)
    g = Solver()
    g.load_model(m)
    g.build_pattern()
    g.assemble(_abi.FP64)
    g.assemble(_abi.FP32)
    x = np.random.default_rng(3).normal(size=m.ndof)
    y = s.matvec(x)
    y64 = g.matvec(x, _abi.FP64)
    y32 = g.matvec(x, _abi.FP32)
    assert np.linalg.norm(y64 - y) <= 1e-12 * np.linalg.norm(y)
    assert np.linalg.norm(y32 - y) <= 1e-5 * np.linalg.norm(y)


def _truth(oracle, m):
    s = _oracle_system(oracle, m)
    rc, u, st = s.solve(eps=1e-14, maxit=200000)
    assert rc in (0, oracle.ERR_MAXIT)
    return s, u


@pytest.mark.parametrize("name", ["quad4", "hex8", "rve", "heat2d"])
def test_fp64_pcg_reference_rule(oracle, name):
    """Same algorithm and stop rule (sqrt(r.r/x.x) < eps) as sparse.cpp."""
    m = MODELS[name]()
    s = _oracle_system(oracle, m)
    rc, u_ref, st_ref = s.solve(eps=1e-10, maxit=100000)
    assert rc == 0
    g = Solver()
    g.load_model(m)
    g.build_pattern()
    g.assemble(_abi.FP64)
    rc, st = g.solve(opts(mode=_abi.MODE_FP64, stop_rule=_abi.STOP_REF, tol=1e-10, maxit=100000, check_every=4))
    u = g.download()
    assert abs(st.iterations - st_ref.iterations) <= max(2, 0.02 * st_ref.iterations)
    _, u_t = _truth(oracle, m)
    err_gpu = np.linalg.norm(u - u_t) / np.linalg.norm(u_t)
    err_ref = np.linalg.norm(u_ref - u_t) / np.linalg.norm(u_t)
    assert err_gpu <= max(10 * err_ref, 1e-12)


@pytest.mark.parametrize("name", ["quad4", "hex8", "rve", "heat2d"])
@pytest.mark.parametrize("precond", [_abi.PRECOND_JACOBI, _abi.PRECOND_BLOCK_JACOBI])
def test_mpir_reaches_1e8(oracle, name, precond):
    m = MODELS[name]()
    _, u_t = _truth(oracle, m)
    g = Solver()
    g.load_model(m)
    g.build_pattern()
    g.assemble(_abi.FP32)
    rc, st = g.solve(opts(mode=_abi.MODE_MPIR, precond=precond, tol=1e-12, inner_tol=0.01, check_every=4))
    u = g.download()
    err = np.linalg.norm(u - u_t) / np.linalg.norm(u_t)
    assert err <= 1e-8, (err, st.as_dict())
    assert st.outer_iterations >= 1
    assert st.true_rel_residual <= 1e-11


def test_fp64_rb_rule_reaches_1e8(oracle):
    m = MODELS["hex8"]()
    _, u_t = _truth(oracle, m)
    g = Solver()
    g.load_model(m)
    g.build_pattern()
    g.assemble(_abi.FP64)
    rc, st = g.solve(opts(mode=_abi.MODE_FP64, stop_rule=_abi.STOP_RB, tol=1e-12, check_every=4))
    u = g.download()
    assert np.linalg.norm(u - u_t) / np.linalg.norm(u_t) <= 1e-8
    assert st.true_rel_residual <= 1e-11


def test_internal_force_matches_oracle(oracle):
    m = MODELS["hex8"]()
    u = np.random.default_rng(2).normal(size=m.ndof)
    f_ref = oracle.internal_force_hex8(m, m.params, m.order, u)
    g = Solver()
    g.load_model(m)
    g.build_pattern()
    f = g.internal_force(u)
    assert np.linalg.norm(f - f_ref) <= 1e-12 * np.linalg.norm(f_ref)


@pytest.mark.parametrize("mode", [_abi.MODE_FP64, _abi.MODE_MPIR])
def test_heat_steps_match_oracle(oracle, mode):
    m = W.heat_slab(10, 8, 6, order=3)
    u0 = m.meta["u0"]
    dt = 1e-3
    s = oracle.System(m)
    s.set_bc(m.restrained, m.prescribed, m.load)
    s.build_pattern()
    u_ref = u0.copy()
    for _ in range(3):
        s.set_bc(m.restrained, m.prescribed, m.load)
        rc, u_ref, st = s.heat_step(m.params, m.order, dt, u_ref, eps=1e-14, maxit=100000)
        assert rc == 0
    g = Solver()
    g.load_model(m)
    g.build_pattern()
    g.heat_set_state(u0)
    st, tot = g.heat_run(dt, 3, opts(mode=mode, tol=1e-13, inner_tol=0.01, check_every=4))
    u = g.heat_get_state()
    assert np.linalg.norm(u - u_ref) / np.linalg.norm(u_ref) <= 1e-8
    assert tot > 0


@pytest.mark.parametrize("mode", [_abi.MODE_FP64, _abi.MODE_MPIR])
def test_quad4_heat_steps_match_oracle(oracle, mode):
    """The 2D transient element (HeatTransferElement2Dtransient) marched
    three backward-Euler steps with a heat input, against the oracle."""
    m = W.heat_plate(16, 11, heat=2.0)
    u0 = m.meta["u0"]
    dt = 1e-3
    s = oracle.System(m)
    s.set_bc(m.restrained, m.prescribed, m.load)
    s.build_pattern()
    u_ref = u0.copy()
    for _ in range(3):
        s.set_bc(m.restrained, m.prescribed, m.load)
        rc, u_ref, st = s.heat_step(m.params, m.order, dt, u_ref, eps=1e-14, maxit=100000)
        assert rc == 0
    g = Solver()
    g.load_model(m)
    g.build_pattern()
    g.heat_set_state(u0)
    st, tot = g.heat_run(dt, 3, opts(mode=mode, tol=1e-13, inner_tol=0.01, check_every=4))
    u = g.heat_get_state()
    assert np.linalg.norm(u - u_ref) / np.linalg.norm(u_ref) <= 1e-8
    assert tot > 0


def _slab_with_top_flux(nx=10, ny=8, nz=6):
    """Diffusion slab held at T = 0 on x = 0 and x = lx only, heated by a
    nodal flux q = 5 + 3x on its top face (SurfaceLoad::applyTo loads)."""
    from betanoox_b200 import surface_flux_load
    m = W.heat_slab(nx, ny, nz, order=3)
    x = m.xyz[:, 0]
    rest = (np.isclose(x, 0.0) | np.isclose(x, x.max())).astype(np.uint8)
    m.restrained = rest
    m.prescribed = np.zeros(m.ndof)
    ztop = m.xyz[:, 2].max()
    faces = m.conn[:, [3, 2, 6, 7]]  # hex8 face zeta = +1 (BETA node order)
    faces = faces[np.all(np.isclose(m.xyz[faces, 2], ztop), axis=1)]
    assert len(faces) == nx * ny
    load = surface_flux_load(faces, m.xyz, 5.0 + 3.0 * x, m.first_dof, m.ndof)
    load[rest.astype(bool)] = 0.0  # the restrained nodes' value is prescribed
    m.load = load
    u0 = m.meta["u0"].copy()
    u0[rest.astype(bool)] = 0.0
    return m, u0


@pytest.mark.parametrize("mode", [_abi.MODE_FP64, _abi.MODE_MPIR])
def test_heat_steps_with_surface_flux_match_oracle(oracle, mode):
    m, u0 = _slab_with_top_flux()
    assert np.abs(m.load).max() > 0
    dt = 1e-3
    s = oracle.System(m)
    s.set_bc(m.restrained, m.prescribed, m.load)
    s.build_pattern()
    u_ref = u0.copy()
    for _ in range(3):
        s.set_bc(m.restrained, m.prescribed, m.load)
        rc, u_ref, st = s.heat_step(m.params, m.order, dt, u_ref, eps=1e-14, maxit=100000)
        assert rc == 0
    g = Solver()
    g.load_model(m)
    g.build_pattern()
    g.heat_set_state(u0)
    st, tot = g.heat_run(dt, 3, opts(mode=mode, tol=1e-13, inner_tol=0.01, check_every=4))
    u = g.heat_get_state()
    assert np.linalg.norm(u - u0) > 1e-3 * np.linalg.norm(u0)  # the flux heats the slab
    assert np.linalg.norm(u - u_ref) / np.linalg.norm(u_ref) <= 1e-8


def test_csr_device_pcg(oracle):
    import torch
    m = MODELS["quad4"]()
    s, u_t = _truth(oracle, m)
    rp, col, val = s.export_lower()
    n = m.ndof
    A = np.zeros((n, n))
    for i in range(n):
        A[i, col[rp[i]:rp[i + 1]]] = val[rp[i]:rp[i + 1]]
    A = A + np.tril(A, -1).T
    import scipy.sparse as sp
    Acsr = sp.csr_matrix(A)
    dev = torch.device("cuda:0")
    d_rp = torch.tensor(Acsr.indptr.astype(np.int32), device=dev)
    d_ci = torch.tensor(Acsr.indices.astype(np.int32), device=dev)
    d_v = torch.tensor(Acsr.data, device=dev, dtype=torch.float64)
    d_b = torch.tensor(s.rhs(), device=dev, dtype=torch.float64)
    d_x = torch.zeros(n, device=dev, dtype=torch.float64)
    lib = _abi.load()
    st = _abi.SolveStats()
    torch.cuda.synchronize()
    rc = lib.beta_gpu_csr_pcg_device(n, d_rp.data_ptr(), d_ci.data_ptr(), d_v.data_ptr(), d_b.data_ptr(),
                                     d_x.data_ptr(), _abi.STOP_RB, 1e-13, 100000, None, C.byref(st))
    assert rc == 0, st.as_dict()
    u = d_x.cpu().numpy()
    assert np.linalg.norm(u - u_t) / np.linalg.norm(u_t) <= 1e-8


# ---- error behaviour (host-made failures; no device fault) ----------------
def test_inverted_element_is_negative_diagonal():
    m = W.cube_hex8(3)
    conn = m.conn.copy()
    conn[4] = conn[4][[4, 5, 6, 7, 0, 1, 2, 3]]  # mirror one element: detJ < 0
    m.conn = conn
    g = Solver()
    g.load_model(m)
    g.build_pattern()
    with pytest.raises(_abi.BetaGpuError) as e:
        g.assemble(_abi.FP64)
    assert e.value.status == _abi.ERR_NEGDIAG


def test_nonfinite_and_bad_inputs_are_rejected():
    m = W.cube_hex8(2)
    g = Solver()
    p = m.params.copy()
    p[0, 0] = np.nan
    with pytest.raises(_abi.BetaGpuError) as e:
        g.load_model(m, params=p)
    assert e.value.status == _abi.ERR_NOT_FINITE
    load = m.load.copy()
    load[0] = 1.0  # dof 0 is clamped
    g2 = Solver()
    g2.load_model(W.cube_hex8(2))
    with pytest.raises(_abi.BetaGpuError) as e:
        g2.set_bc(m.restrained, m.prescribed, load)
    assert e.value.status == _abi.ERR_LOAD_ON_RESTRAINED


def test_maxit_is_reported_not_fatal():
    m = MODELS["hex8"]()
    g = Solver()
    g.load_model(m)
    g.build_pattern()
    g.assemble(_abi.FP64)
    rc, st = g.solve(opts(mode=_abi.MODE_FP64, tol=1e-14, maxit=3, check_every=1), raise_on_error=False)
    assert rc == _abi.MAXIT and st.iterations == 3
    # the context stays usable
    rc, st = g.solve(opts(mode=_abi.MODE_FP64, tol=1e-10, check_every=8))
    assert rc == 0


@pytest.mark.parametrize("name", ["rve", "quad4"])
def test_element_outputs_match_oracle(oracle, name):
    """Post-solve volume integrals (getVolAvgValues) of the solved field."""
    m = MODELS[name]()
    g = Solver()
    g.load_model(m)
    g.build_pattern()
    g.assemble(_abi.FP32)
    g.solve(opts(tol=1e-12))
    u = g.download()
    per, tot = g.element_outputs()
    ref = oracle.element_outputs(m, m.params, m.order, u)
    scale = np.abs(ref).max(axis=0)
    scale[scale == 0] = 1.0
    assert (np.abs(per - ref) / scale).max() <= 1e-12
    np.testing.assert_allclose(tot, per.sum(axis=0), rtol=1e-12, atol=1e-300)
    per2, _ = g.element_outputs(u)  # explicit displacements give the same
    np.testing.assert_array_equal(per, per2)
