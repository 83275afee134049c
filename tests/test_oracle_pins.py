"""The oracle pinned against the reference's own code and known answers.

* Gauss points/weights and shape functions vs the reference's gauss.cpp and
  shape.cpp (golden vectors produced by those files, tests/golden).
* Dense LU inverse vs the known answer in the reference's matrix.cpp debug main.
* Analytic element properties the reference's elements must satisfy.
* Element matrices, constitutive matrices and the global assembly and solve
  against the reference's own element, material and Equations code compiled
  unmodified (oracle/_ref), through committed golden vectors and, where that
  build exists, live.
"""
import importlib.util
import json
import os

import numpy as np
import pytest

from betanoox_b200 import workloads as W

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _load(name):
    with open(os.path.join(GOLD, name)) as f:
        return json.load(f)


def _gen_golden():
    """The fixture generator, for the cases it defines (it imports the oracle
    and the workloads, nothing from the reference at import time)."""
    spec = importlib.util.spec_from_file_location("gen_golden", os.path.join(GOLD, "gen_golden.py"))
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    return gen


def test_gauss_matches_reference_golden(oracle):
    g = _load("ref_quadrature.json")
    for k, d in g["gauss"].items():
        x, w = oracle.gauss_1d(int(k))
        np.testing.assert_array_equal(x, np.array(d["x"]))  # same Newton recurrence: bit-exact
        np.testing.assert_array_equal(w, np.array(d["w"]))


def test_tensor_points_match_reference_golden(oracle):
    g = _load("ref_quadrature.json")
    for o, d in g["hex"].items():
        xi, eta, zeta, w = oracle.hex_points(int(o))
        for a, key in ((xi, "xi"), (eta, "eta"), (zeta, "zeta"), (w, "w")):
            np.testing.assert_array_equal(a, np.array(d[key]))
    for o, d in g["quad"].items():
        xi, eta, w = oracle.quad_points(int(o))
        for a, key in ((xi, "xi"), (eta, "eta"), (w, "w")):
            np.testing.assert_array_equal(a, np.array(d[key]))


def test_shape_functions_match_reference_golden(oracle):
    g = _load("ref_quadrature.json")
    for d in g["shape_hex8"]:
        S, d0, d1, d2 = oracle.shape_hex8(*d["at"])
        for a, key in ((S, "S"), (d0, "dxi"), (d1, "deta"), (d2, "dzeta")):
            np.testing.assert_allclose(a, np.array(d[key]), rtol=0, atol=1e-15)
    for d in g["shape_quad4"]:
        S, d0, d1 = oracle.shape_quad4(*d["at"])
        for a, key in ((S, "S"), (d0, "dxi"), (d1, "deta")):
            np.testing.assert_allclose(a, np.array(d[key]), rtol=0, atol=1e-15)


def test_reference_leaf_live_if_present(oracle):
    """When oracle/_ref was built here, compare against it directly as well."""
    if not oracle.RefLeaf.available():
        pytest.skip("oracle/_ref not built (reference tree absent)")
    r = oracle.RefLeaf()
    for k in range(1, 12):
        x, w = oracle.gauss_1d(k)
        xr, wr = r.gauss_1d(k)
        np.testing.assert_array_equal(x, xr)
        np.testing.assert_array_equal(w, wr)
    rng = np.random.default_rng(0)
    for p in rng.uniform(-1, 1, size=(50, 3)):
        a = oracle.shape_hex8(*p)
        b = r.shape_hex8(*p)
        for u, v in zip(a, b):
            np.testing.assert_allclose(u, v, rtol=0, atol=1e-15)


def test_matrix_invert_kat(oracle):
    k = _load("ref_matrix_kat.json")
    inv = oracle.invert(np.array(k["B"], float))
    np.testing.assert_allclose(inv, np.array(k["B_inverse"]), rtol=0, atol=10 ** -k["B_inverse_digits"])
    A = np.array(k["A"], float)
    B = np.array(k["B"], float)
    np.testing.assert_array_equal(A @ B, np.array(k["A_times_B"]))
    np.testing.assert_array_equal(A + B, np.array(k["A_plus_B"]))


def _unit_hex(scale=(1.0, 1.0, 1.0), jitter=0.0):
    xyz = np.array([[0, 0, 0], [0, 1, 0], [0, 1, 1], [0, 0, 1], [1, 0, 0], [1, 1, 0], [1, 1, 1], [1, 0, 1]], float)
    return xyz * np.array(scale) + jitter * np.sin(np.arange(24).reshape(8, 3))


def test_hex8_rigid_modes_and_symmetry(oracle):
    xyz = _unit_hex((0.8, 1.2, 0.9), 0.07)
    C = oracle.cmat_ortho3d(W.iso3d_params(np.array([1e4]), 0.3)[0])
    st, K = oracle.ke_hex8(xyz, C, 2)
    assert st == 0
    np.testing.assert_allclose(K, K.T, rtol=0, atol=1e-9 * np.abs(K).max())
    # six rigid-body modes lie in the null space
    modes = []
    for c in range(3):
        m = np.zeros((8, 3)); m[:, c] = 1; modes.append(m.ravel())
    for (i, j) in ((0, 1), (1, 2), (0, 2)):
        m = np.zeros((8, 3)); m[:, i] = -xyz[:, j]; m[:, j] = xyz[:, i]; modes.append(m.ravel())
    for m in modes:
        assert np.abs(K @ m).max() < 1e-9 * np.abs(K).max()
    ev = np.linalg.eigvalsh(K)
    assert (ev[6:] > 1e-8 * ev[-1]).all()


def test_hex8_constant_strain_patch(oracle):
    """A linear displacement field gives Fe = K u consistent with uniform stress."""
    xyz = _unit_hex((1.0, 1.0, 1.0), 0.05)
    C = oracle.cmat_ortho3d(W.iso3d_params(np.array([200.0]), 0.25)[0])
    grad = np.array([[1e-3, 2e-4, 0], [0, -5e-4, 1e-4], [3e-4, 0, 2e-3]])
    u = (xyz @ grad.T).ravel()
    st, K = oracle.ke_hex8(xyz, C, 2)
    fe = oracle.fe_hex8(xyz, C, u, 2)
    np.testing.assert_allclose(K @ u, fe, rtol=1e-12, atol=1e-15)


def test_quad4_and_heat_properties(oracle):
    xy = np.array([[0, 0], [1.2, 0.1], [1.0, 0.9], [-0.1, 1.0]], float)
    st, K = oracle.ke_quad4(xy, oracle.cmat_plane_stress(W.pstress_params(np.array([70e3]), 0.3)[0]), 2)
    assert st == 0
    for m in (np.tile([1, 0], 4), np.tile([0, 1], 4), np.stack([-xy[:, 1], xy[:, 0]], 1).ravel()):
        assert np.abs(K @ m).max() < 1e-9 * np.abs(K).max()
    xyz = _unit_hex((0.5, 0.7, 0.3), 0.02)
    st, Kh, Mh = oracle.km_hex8_heat(xyz, [1.0, 2.0, 3.0], 1.5, 3)
    assert np.abs(Kh @ np.ones(8)).max() < 1e-12 * np.abs(Kh).max()
    # sum of the consistent capacity matrix = c * volume
    vol = 0.0
    xi, eta, zeta, w = oracle.hex_points(3)
    for p in range(len(w)):
        _, d0, d1, d2 = oracle.shape_hex8(xi[p], eta[p], zeta[p])
        J = np.stack([d0 @ xyz, d1 @ xyz, d2 @ xyz])
        vol += np.linalg.det(J) * w[p]
    assert abs(Mh.sum() - 1.5 * vol) < 1e-12


def test_small_system_solves_to_reference_rule(oracle):
    m = W.plate_quad4(8)
    s = oracle.System(m)
    assert s.set_bc(m.restrained, m.prescribed, m.load) == 0
    s.build_pattern()
    assert s.assemble(m.params, m.order) == 0
    rc, u, st = s.solve(eps=1e-10, maxit=10000)
    assert rc == 0 and st.last_norm < 1e-10
    # the lower-triangle product equals the full symmetric product
    rp, col, val = s.export_lower()
    n = m.ndof
    A = np.zeros((n, n))
    for i in range(n):
        for k in range(rp[i], rp[i + 1]):
            A[i, col[k]] = val[k]
            A[col[k], i] = val[k]
    x = np.random.default_rng(1).normal(size=n)
    np.testing.assert_allclose(s.matvec(x), A @ x, rtol=1e-13, atol=1e-12)
    b = s.rhs()
    np.testing.assert_allclose(A @ u, b, rtol=0, atol=1e-8 * np.abs(b).max())


def test_load_on_restrained_is_an_error(oracle):
    m = W.plate_quad4(4)
    load = m.load.copy()
    load[0] = 1.0  # dof 0 belongs to the clamped left edge
    s = oracle.System(m)
    assert s.set_bc(m.restrained, m.prescribed, load) == oracle.ERR_LOAD_ON_RESTRAINED


def test_oracle_threaded_pcg_matches_serial(oracle):
    m = W.cube_hex8(5, seed=3)
    s = oracle.System(m)
    s.set_bc(m.restrained, m.prescribed, m.load)
    s.build_pattern()
    s.assemble(m.params, m.order)
    b = s.rhs()
    rc1, u1, st1 = s.solve(eps=1e-12, maxit=20000)
    rc2, u2, st2 = s.solve_threaded(b, eps=1e-12, maxit=20000, threads=4)
    assert rc1 == 0 and rc2 == 0
    assert np.linalg.norm(u1 - u2) / np.linalg.norm(u1) < 1e-9


def test_element_outputs_known_answer_for_a_uniform_strain(oracle):
    """getVolAvgValues under u = H x (a uniform strain): every element's
    strain integral is E V, its stress integral C E V and its energy
    0.5 E.C E V -- exact for any element shape and material."""
    rng = np.random.default_rng(11)
    m = W.cube_hex8(3, seed=8)
    m.xyz = m.xyz + 0.05 * rng.uniform(-1, 1, size=m.xyz.shape) / 3  # distorted hexes
    H = rng.normal(size=(3, 3)) * 1e-3
    u = (m.xyz @ H.T).reshape(-1)
    E = np.array([H[0, 0], H[1, 1], H[2, 2], H[0, 1] + H[1, 0], H[1, 2] + H[2, 1], H[0, 2] + H[2, 0]])
    out = oracle.element_outputs(m, m.params, m.order, u)
    for e in range(m.nelem):
        C = oracle.cmat_ortho3d(m.params[e])
        V = out[e, 0]
        np.testing.assert_allclose(out[e, 7:13], E * V, rtol=1e-9, atol=1e-18)
        np.testing.assert_allclose(out[e, 1:7], C @ E * V, rtol=1e-9, atol=1e-12)
        assert abs(out[e, 13] - 0.5 * E @ C @ E * V) <= 1e-9 * abs(0.5 * E @ C @ E * V)
    q = W.plate_quad4(4)
    Hq = rng.normal(size=(2, 2)) * 1e-3
    uq = (q.xyz @ Hq.T).reshape(-1)
    Eq = np.array([Hq[0, 0], Hq[1, 1], Hq[0, 1] + Hq[1, 0]])
    outq = oracle.element_outputs(q, q.params, q.order, uq)
    assert abs(outq[:, 0].sum() - 1.0) < 1e-12  # undistorted unit square
    Cq = oracle.cmat_plane_stress(q.params[0])
    np.testing.assert_allclose(outq[:, 4:7].sum(axis=0), Eq, rtol=1e-9)
    np.testing.assert_allclose(outq[:, 1:4].sum(axis=0), Cq @ Eq, rtol=1e-9)


def test_quad4_diffusion_known_answers(oracle):
    """2D transient element on the unit square, k = 1, c = 2: the bilinear
    conductivity (4, -1, -2, -1)/6 and consistent capacity c A (4, 2, 1, 2)/36
    patterns; K annihilates constants; anisotropy and scaling as they must."""
    sq = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], dtype=float)
    st, K, M = oracle.km_quad4_heat(sq, (1.0, 1.0), 2.0, order=2)
    assert st == 0
    k_row = np.array([4, -1, -2, -1]) / 6.0
    m_row = 2.0 * np.array([4, 2, 1, 2]) / 36.0
    for i in range(4):
        np.testing.assert_allclose(K[i], np.roll(k_row, i), atol=1e-15)
        np.testing.assert_allclose(M[i], np.roll(m_row, i), atol=1e-15)
    # a rectangle 3 x 0.5 with k11 = 2, k22 = 5: K x-part scales by k11 h/w, y-part by k22 w/h
    rect = sq * np.array([3.0, 0.5])
    _, K2, M2 = oracle.km_quad4_heat(rect, (2.0, 5.0), 1.0, order=3)
    assert np.abs(K2 @ np.ones(4)).max() <= 1e-13
    assert abs(M2.sum() - 1.5) <= 1e-13  # c * area
    kx = 2.0 * 0.5 / 3.0 * np.array([[2, -2, -1, 1], [-2, 2, 1, -1], [-1, 1, 2, -2], [1, -1, -2, 2]]) / 6.0
    ky = 5.0 * 3.0 / 0.5 * np.array([[2, 1, -1, -2], [1, 2, -2, -1], [-1, -2, 2, 1], [-2, -1, 1, 2]]) / 6.0
    np.testing.assert_allclose(K2, kx + ky, atol=1e-12)


_CG_MODELS = {"plate_quad4_12": lambda: W.plate_quad4(12), "cube_hex8_5_s3": lambda: W.cube_hex8(5, seed=3),
              "heat_plate_12x9": lambda: W.heat_plate(12, 9, heat=2.0)}


@pytest.mark.parametrize("name", list(_CG_MODELS))
def test_oracle_pcg_matches_the_reference_cg(oracle, name, tmp_path):
    """The oracle's Jacobi-PCG against the reference's own
    SymmetricSparseMatrix::solve (sparse.cpp, compiled unmodified): the same
    iteration count and the same solution, on the reference's golden outputs
    and, where oracle/_ref is built, live on the matrix written in the
    lower-triangle address format and read by the reference's own reader."""
    case = {c["name"]: c for c in _load("ref_cg.json")["cases"]}[name]
    m = _CG_MODELS[name]()
    s = oracle.System(m)
    s.set_bc(m.restrained, m.prescribed, m.load)
    s.build_pattern()
    s.assemble(m.params, m.order)
    rc, x, st = s.solve(eps=case["eps"], maxit=100000)
    assert rc == 0
    xr = np.array(case["x"])
    assert st.iterations == case["iterations"]
    assert np.abs(x - xr).max() <= 1e-12 * np.abs(xr).max()
    if oracle.RefLeaf.available():
        from betanoox_b200 import _abi, write_lower
        rp, col, val = s.export_lower()
        p = tmp_path / "k.txt"
        write_lower(p, _abi.FMT_ADDRESS_LOWER, rp, col, val)
        x_live, it_live = oracle.RefLeaf().sparse_solve_file(p, s.rhs(), case["eps"])
        assert it_live == st.iterations
        assert np.abs(x_live - x).max() <= 1e-12 * np.abs(x).max()


def test_quad4_diffusion_equals_the_reference_addToKe(oracle):
    """The oracle's 2D diffusion conductivity against the reference's own
    HeatTransferElement2Dtransient::addToKe (compiled unmodified),
    accumulated over the reference's Gauss points on a distorted quad."""
    case = _load("ref_quadrature.json")["heat2d_ke"]
    xy = np.array(case["xy"])
    iu = np.triu_indices(4)
    for order, Kref in case["orders"].items():
        st, K, _ = oracle.km_quad4_heat(xy, (case["k11"], case["k22"]), 1.0, order=int(order))
        assert st == 0
        Kref = np.array(Kref)
        assert np.abs(K[iu] - Kref[iu]).max() <= 1e-14 * np.abs(Kref).max()


def test_hex8_diffusion_equals_the_reference_element(oracle):
    """The oracle's hex8 diffusion K (full anisotropic conductivity) and M,
    and the step's Mbar = (a1 K + M)/dt and F = -(a1+a2)/dt K u_s, against
    the reference's own HeatTransferElement3Dtransient::addToKe, addToMe,
    formK_s and formF_s_new (compiled unmodified) on a distorted hex8."""
    case = _load("ref_quadrature.json")["heat3d"]
    X, k9 = np.array(case["xyz"]), np.array(case["k9"])
    iu = np.triu_indices(8)
    for order, ref in case["orders"].items():
        st, K, M = oracle.km_hex8_heat(X, k9, case["cap"], order=int(order))
        assert st == 0
        Kr, Mr = np.array(ref["K"]), np.array(ref["M"])
        assert np.abs(K[iu] - Kr[iu]).max() <= 1e-14 * np.abs(Kr).max()
        assert np.abs(M[iu] - Mr[iu]).max() <= 1e-14 * np.abs(Mr).max()
        # the step terms, from the upper triangles as the reference keeps them
        Ku, Mu = np.triu(K), np.triu(M)
        mbar = (case["a1"] * Ku + Mu) / case["dt"]
        f = -(case["a1"] + case["a2"]) / case["dt"] * (K @ np.array(case["u_s"]))
        assert np.abs(mbar - np.array(ref["Mbar"])).max() <= 1e-14 * np.abs(mbar).max()
        assert np.abs(f - np.array(ref["F"])).max() <= 1e-13 * np.abs(f).max()


def _ref_elastic_hex8(r, X, C6, u, order):
    xi, eta, zeta, w = r.hex_points(order)
    K, F = np.zeros((24, 24)), np.zeros(24)
    for a, b, c, wt in zip(xi, eta, zeta, w):
        S, d0, d1, d2 = r.shape_hex8(a, b, c)
        J = np.array([d0 @ X, d1 @ X, d2 @ X])
        g = np.linalg.solve(J, np.array([d0, d1, d2]))
        K, F, _ = r.elastic_point(C6, g[0], g[1], g[2], np.linalg.det(J) * wt, K, u=u, Fe=F)
    return K, F


def test_elasticity_equals_the_reference_elements(oracle):
    """The oracle's hex8 stiffness and internal force and its quad4 plane
    stiffness, for general (anisotropic) constitutive matrices, against the
    reference's own ElasticityElement3D (calculateBmatrix, addToKe,
    derivativesOfFields, calculateStrain, addToFe) and ElasticityElement2D
    (calculateBmatrix, addToKe), compiled unmodified, summed over the
    reference's Gauss points on distorted elements."""
    g = _load("ref_quadrature.json")
    case = g["elastic3d"]
    X, C6, u = np.array(case["xyz"]), np.array(case["C"]), np.array(case["u"])
    iu = np.triu_indices(24)
    for order, ref in case["orders"].items():
        st, K = oracle.ke_hex8(X, C6, order=int(order))
        assert st == 0
        Kr, Fr = np.array(ref["K"]), np.array(ref["F"])
        assert np.abs(K[iu] - Kr[iu]).max() <= 1e-14 * np.abs(Kr).max()
        F = oracle.fe_hex8(X, C6, u, order=int(order))
        assert np.abs(F - Fr).max() <= 1e-14 * np.abs(Fr).max()
    case = g["elastic2d"]
    X2, C3 = np.array(case["xy"]), np.array(case["C"])
    iu = np.triu_indices(8)
    for order, ref in case["orders"].items():
        st, K = oracle.ke_quad4(X2, C3, order=int(order))
        assert st == 0
        Kr = np.array(ref["K"])
        assert np.abs(K[iu] - Kr[iu]).max() <= 1e-14 * np.abs(Kr).max()
    if oracle.RefLeaf.available():
        # live, on further random elements and the oracle's own D matrices
        r = oracle.RefLeaf()
        rng = np.random.default_rng(11)
        base = np.array([[0, 0, 0], [0, 1, 0], [0, 1, 1], [0, 0, 1], [1, 0, 0], [1, 1, 0], [1, 1, 1], [1, 0, 1]],
                        float)
        for trial in range(3):
            X = base * rng.uniform(0.5, 2.0, 3) + rng.uniform(-0.1, 0.1, (8, 3))
            C6 = oracle.cmat_ortho3d([rng.uniform(50, 200), rng.uniform(5, 20), rng.uniform(5, 20),
                                      0.25, 0.3, 0.28, 4.0, 3.0, 5.0])
            u = rng.normal(size=24)
            Kr, Fr = _ref_elastic_hex8(r, X, C6, u, 2)
            st, K = oracle.ke_hex8(X, C6, order=2)
            assert np.abs(K[np.triu_indices(24)] - Kr[np.triu_indices(24)]).max() <= 1e-14 * np.abs(Kr).max()
            F = oracle.fe_hex8(X, C6, u, order=2)
            assert np.abs(F - Fr).max() <= 1e-14 * np.abs(Fr).max()


def test_constitutive_matrices_equal_the_reference_materials(oracle):
    """The oracle's 3D orthotropic stiffness (compliance filled from the nine
    constants, then inverted) and plane-stress stiffness are bit-identical to
    what the reference's own ElasticMaterial::read (readModuli) and
    PlaneStress::read build, compiled unmodified with its Matrix::invert, and
    the oracle's dense inverse (the same Crout factorisation) is
    bit-identical to Matrix::invert."""
    g = _load("ref_materials.json")
    for case in g["ortho3d"]:
        np.testing.assert_array_equal(oracle.cmat_ortho3d(case["m9"]), np.array(case["C"]))
    for case in g["plane_stress"]:
        np.testing.assert_array_equal(oracle.cmat_plane_stress(case["m4"]), np.array(case["C"]))
    for case in g["invert"]:
        np.testing.assert_array_equal(oracle.invert(np.array(case["A"])), np.array(case["inverse"]))
    if oracle.RefMaterial.available():
        r = oracle.RefMaterial()
        rng = np.random.default_rng(5)
        for _ in range(20):
            e = rng.uniform(1.0, 300.0, 3)
            m9 = [e[0], e[1], e[2], rng.uniform(0.1, 0.35), rng.uniform(0.1, 0.35), rng.uniform(0.1, 0.35),
                  *rng.uniform(1.0, 50.0, 3)]
            C = oracle.cmat_ortho3d(m9)
            np.testing.assert_array_equal(C, r.cmat_ortho3d(m9))
            eps = rng.normal(size=6)
            assert np.abs(C @ eps - r.elastic_stress(m9, eps)).max() <= 1e-14 * np.abs(C @ eps).max()
            m4 = [e[0], e[1], m9[3], m9[6]]
            np.testing.assert_array_equal(oracle.cmat_plane_stress(m4), r.cmat_plane_stress(m4))
            A = rng.normal(size=(7, 7))
            np.testing.assert_array_equal(oracle.invert(A), r.invert(A))


def _oracle_system(oracle, m, solve, eps):
    s = oracle.System(m)
    assert s.set_bc(m.restrained, m.prescribed, m.load) == 0
    s.build_pattern()
    assert s.assemble(m.params, m.order) == 0
    rp, col, val = s.export_lower()
    x = s.solve(eps=eps, maxit=10000)[1] if solve else None
    return rp, col, val, s.pseudo_load(), x


def test_global_assembly_equals_the_reference_equations(oracle):
    """The oracle's global system -- lower-triangle pattern, assembled values
    with the restraint elimination, pseudo-load vector and CG solution -- is
    bit-identical to the reference's own Equations (equation.cpp:
    specifyNonZeroLocation, allocate, addMatrix, addLoadToEqn, solve over
    sparse.cpp's SymmetricSparseMatrix, compiled unmodified) given the same
    element matrices: on renumbered meshes, with nonzero prescribed
    displacements, an unused node, elasticity and diffusion."""
    gen = _gen_golden()
    EQUATION_CASES, element_maps = gen.EQUATION_CASES, gen.element_maps
    g = _load("ref_equations.json")
    for name, make in EQUATION_CASES.items():
        ref = g["cases"][name]
        m = make()
        rp, col, val, pseudo, x = _oracle_system(oracle, m, ref["x"] is not None, g["eps"])
        np.testing.assert_array_equal(rp, np.array(ref["rowptr"]))
        np.testing.assert_array_equal(col, np.array(ref["col"]))
        np.testing.assert_array_equal(val, np.array(ref["val"]))
        np.testing.assert_array_equal(pseudo, np.array(ref["pseudo"]))
        if x is not None:
            np.testing.assert_allclose(x, np.array(ref["x"]), rtol=0, atol=1e-14 * np.abs(x).max())
    if oracle.RefEquations.available():
        r = oracle.RefEquations()
        for m, solve in ((W.renumbered(W.cube_hex8(3, seed=4), 9, unused_node=True), False),
                         (W.renumbered(W.rve_hex8(3, seed=2), 5), True)):
            nd = m.nnpe * m.ndpn
            st, Ke = oracle.element_matrices_threaded(m, m.params, m.order, 0, m.nelem)
            got = r.assemble(m.ndof, element_maps(m), Ke.reshape(m.nelem, nd, nd), m.restrained, m.prescribed,
                             m.load, solve=solve, eps=1e-10)
            rp, col, val, pseudo, x = _oracle_system(oracle, m, solve, 1e-10)
            for a, b in ((rp, got[0]), (col, got[1]), (val, got[2]), (pseudo, got[3])):
                np.testing.assert_array_equal(a, b)
            if solve:
                np.testing.assert_allclose(x, got[5], rtol=0, atol=1e-14 * np.abs(x).max())


def test_transient_steps_equal_the_reference_step(oracle):
    """Three backward-Euler steps of a hex8 slab (alpha 1 and 0.5, with and
    without a heat input) and of a quad4 plate with a heat input (the 2D
    element, which inherits the step terms): the oracle's heat_step is
    bit-identical to the
    step composed from the reference's own code in DiffusionModel's order
    (DiffusionModel.cpp:743-818, 322-347) -- formK_s / formF_s_new of
    HeatTransferElement3Dtransient per element, Equations::addMatrix of
    Mbar_e with Fbar_e, Equations::solve from u_s, u_s + delta."""
    gen = _gen_golden()
    g = _load("ref_heat_steps.json")
    for name, case in g["cases"].items():
        m = gen.heat_step_case(case["with_load"], case.get("quad4", False))
        s = oracle.System(m)
        s.set_bc(m.restrained, m.prescribed, m.load)
        s.build_pattern()
        u = m.meta["u0"].copy()
        for k in range(g["steps"]):
            s.set_bc(m.restrained, m.prescribed, m.load)
            rc, u, st = s.heat_step(m.params, m.order, g["dt"], u, alpha=case["alpha"], eps=g["eps"], maxit=100000)
            assert rc == 0
            np.testing.assert_array_equal(u, np.array(case["u"][k]), err_msg=f"{name} step {k}")
    if oracle.RefLeaf.available() and oracle.RefEquations.available():
        leaf, req = oracle.RefLeaf(), oracle.RefEquations()
        m = gen.heat_step_case(True)
        s = oracle.System(m)
        s.set_bc(m.restrained, m.prescribed, m.load)
        s.build_pattern()
        u_o = u_r = m.meta["u0"] + 0.1
        for _ in range(2):
            s.set_bc(m.restrained, m.prescribed, m.load)
            rc, u_o, st = s.heat_step(m.params, m.order, 5e-4, u_o, alpha=0.75, eps=1e-14, maxit=100000)
            u_r = gen.ref_heat_step(leaf, req, m, u_r, 5e-4, 0.75, 1e-14)
            np.testing.assert_array_equal(u_o, u_r)


def test_parcg_solves_like_the_oracle(oracle):
    """The reference's two-thread solver (ParCG.cpp ParCGMatrix::solve, the
    same Jacobi-PCG with its dot products split between two OpenMP threads,
    compiled unmodified) reaches the oracle's solution to rounding on a system
    assembled through the reference's Equations."""
    if not oracle.RefEquations.available():
        pytest.skip("oracle/_ref not built (reference tree absent)")
    gen = _gen_golden()
    req = oracle.RefEquations()
    for m in (W.rve_hex8(3, seed=2), W.renumbered(W.cube_hex8(6, seed=1), 4)):
        nd = m.nnpe * m.ndpn
        st, Ke = oracle.element_matrices_threaded(m, m.params, m.order, 0, m.nelem)
        got = req.assemble(m.ndof, gen.element_maps(m), Ke.reshape(m.nelem, nd, nd), m.restrained, m.prescribed,
                           m.load, solve=True, eps=1e-10, maxit=100000, parcg=True)
        x = _oracle_system(oracle, m, True, 1e-10)[4]
        assert np.abs(got[5] - x).max() <= 1e-11 * np.abs(x).max()


def test_internal_force_equals_the_reference_resultant(oracle):
    """The oracle's global internal force (restrained rows skipped) against
    the reference's: element forces from ElasticityElement3D's own
    derivativesOfFields / calculateStrain / addToFe summed by
    Equations::assembleResultantVector (compiled unmodified), on a renumbered
    cube under a random displacement; live, the oracle's element forces
    through the reference's assembleResultantVector are bit-identical."""
    gen = _gen_golden()
    m, u = gen.internal_force_case()
    f = oracle.internal_force_hex8(m, m.params, m.order, u, m.restrained)
    ref = np.array(_load("ref_internal_force.json")["f"])
    assert np.abs(f - ref).max() <= 1e-14 * np.abs(ref).max()
    if oracle.RefEquations.available():
        maps = gen.element_maps(m)
        Fe = np.stack([oracle.fe_hex8(m.xyz[m.conn[e]], oracle.cmat_ortho3d(m.params[e]), u[maps[e]], m.order)
                       for e in range(m.nelem)])
        np.testing.assert_array_equal(oracle.RefEquations().resultant(m.ndof, maps, Fe, m.restrained), f)


def test_zero_diagonal_replacement_equals_the_reference(oracle):
    """LargeMatrix::CheckAndFixZeroDiagonal (largeMatrix.cpp:43-79) through
    the solve: rows of an unused free node hold only a zero diagonal.
    Without a replacement value the oracle refuses (the reference exits);
    with ReplaceZeroDiagonal set, its solution is bit-identical to the
    reference's Equations solve."""
    gen = _gen_golden()
    m = gen.zero_diag_case()
    g = _load("ref_equations.json")["zero_diag"]
    s = oracle.System(m)
    s.set_bc(m.restrained, m.prescribed, m.load)
    s.build_pattern()
    s.assemble(m.params, m.order)
    assert s.solve(eps=1e-10, maxit=10000)[0] == oracle.ERR_ZERO_DIAG
    s.set_zero_diag(g["value"])
    rc, x, st = s.solve(eps=1e-10, maxit=10000)
    assert rc == 0
    np.testing.assert_array_equal(x, np.array(g["x"]))


def test_conductivity_equals_the_reference_material(oracle):
    """HeatTransferMaterial::read of a readConductivity block (the reference's
    own heatTransferMaterial.cpp, compiled unmodified) builds diag(k11, k22,
    k33), the tensor the oracle's diffusion elements take from the same three
    parameters: element matrices from either are bit-identical; its flux is
    -k grad T."""
    xyz = _unit_hex((0.9, 1.1, 0.8), 0.04)
    for case in _load("ref_materials.json")["conductivity"]:
        C9 = np.array(case["C"])
        np.testing.assert_array_equal(C9, np.diag(case["k3"]))
        np.testing.assert_array_equal(np.array(case["flux"]), -(C9 @ np.array(case["grad"])))
        a = oracle.km_hex8_heat(xyz, case["k3"], 1.3, order=2)
        b = oracle.km_hex8_heat(xyz, C9, 1.3, order=2)
        np.testing.assert_array_equal(a[1], b[1])
        np.testing.assert_array_equal(a[2], b[2])


def _one_element_model(kind, X, params):
    nnpe, ndim = X.shape
    ndpn = 3 if kind == 2 else 2
    n = nnpe * ndpn
    return W.Model("one element", kind, ndim, np.ascontiguousarray(X, float), np.arange(nnpe, dtype=np.int32)[None, :],
                   ndpn, np.asarray(params, float)[None, :], np.zeros(n, np.uint8), np.zeros(n), np.zeros(n), 2)


def test_element_driver_and_outputs_equal_the_reference(oracle):
    """The reference's own element driver and post-solve outputs (compiled
    unmodified; isoElement.cpp's interpolation and Jacobian supplied by the
    shim): ElasticityElement3D::update("KF") -- loopOverIntegrationPoints,
    processActionCode, calculateStress / calculateFe / calculateKe -- against
    the oracle's hex8 stiffness and internal force, ElasticityElement2D
    through the same driver against the quad4 stiffness, and getVolAvgValues
    against the oracle's element outputs (volume, stress and strain
    integrals, strain energy)."""
    gen = _gen_golden()
    X, m9, u, X2, m4, u2 = gen.elastic_driver_inputs()
    g = _load("ref_quadrature.json")["elastic_driver"]
    C6, C3 = oracle.cmat_ortho3d(m9), oracle.cmat_plane_stress(m4)
    iu = np.triu_indices(24)
    for order, ref in g["hex8"].items():
        o = int(order)
        Kr, Fr, va = np.array(ref["K"]), np.array(ref["F"]), np.array(ref["vol_avg"])
        K = oracle.ke_hex8(X, C6, o)[1]
        assert np.abs(K[iu] - Kr[iu]).max() <= 1e-14 * np.abs(Kr).max()
        F = oracle.fe_hex8(X, C6, u, o)
        assert np.abs(F - Fr).max() <= 1e-14 * np.abs(Fr).max()
        out = oracle.element_outputs(_one_element_model(2, X, m9), np.asarray(m9)[None, :], o, u)[0]
        ref_row = np.concatenate([va[:13], va[13:14]])  # volume, stress (6), strain (6), SED
        np.testing.assert_allclose(out, ref_row, rtol=1e-13, atol=1e-14 * np.abs(ref_row).max())
    ref = g["quad4"]["2"]
    Kr = np.array(ref["K"])
    iu = np.triu_indices(8)
    K = oracle.ke_quad4(X2, C3, 2)[1]
    assert np.abs(K[iu] - Kr[iu]).max() <= 1e-14 * np.abs(Kr).max()
    out = oracle.element_outputs(_one_element_model(1, X2, m4), np.asarray(m4)[None, :], 2, u2)[0]
    np.testing.assert_allclose(out[:7], np.concatenate([[ref["volume"]], ref["stress"], ref["strain"]]),
                               rtol=1e-13, atol=1e-14)


def test_diffusion_driver_equals_the_reference(oracle):
    """The reference's own diffusion element driver (compiled unmodified):
    HeatTransferElement3Dtransient::update("KM") -- loopOverIntegrationPoints,
    processActionCode, calculateKe / calculateMe -- and the 2D element
    through the same driver, against the oracle's K and M."""
    X, k3, c3, X2, k2, c2 = _gen_golden().heat_driver_inputs()
    g = _load("ref_quadrature.json")["heat_driver"]
    for order in ("2", "3"):
        for key, (st, K, M) in (("hex8", oracle.km_hex8_heat(X, k3, c3, order=int(order))),
                                ("quad4", oracle.km_quad4_heat(X2, k2, c2, order=int(order)))):
            ref = g[key][order]
            Kr, Mr = np.array(ref["K"]), np.array(ref["M"])
            iu = np.triu_indices(Kr.shape[0])
            assert np.abs(K[iu] - Kr[iu]).max() <= 1e-14 * np.abs(Kr).max()
            assert np.abs(M[iu] - Mr[iu]).max() <= 1e-14 * np.abs(Mr).max()


def test_dof_numbering_and_node_records_equal_the_reference(oracle, abi, tmp_path):
    """Node::setNumDofPerNode (node.cpp, compiled unmodified): a uniform
    "n all" block numbers dofs node-major, firstDof = n * node -- the
    numbering the library and the workloads use -- and mixed blocks give the
    running sum; the node records of the library's binary mesh writer are
    byte-identical to Node::writeBinary's, and Node::readBinary reads them."""
    if not oracle.RefMaterial.available():
        pytest.skip("oracle/_ref not built (reference tree absent)")
    r = oracle.RefMaterial()
    m = W.cube_hex8(3, seed=1)
    nd, fd, tot = r.set_num_dof(m.nnode, "3 all\nend\n")
    assert (nd == 3).all() and tot == m.ndof
    np.testing.assert_array_equal(fd, m.first_dof)
    nd, fd, tot = r.set_num_dof(10, "2 0 9 1\n3 1 9 2\nend\n")
    np.testing.assert_array_equal(nd, [2, 3, 2, 3, 2, 3, 2, 3, 2, 3])
    np.testing.assert_array_equal(fd, np.concatenate([[0], np.cumsum(nd)[:-1]]))
    assert tot == nd.sum()
    xyz = np.ascontiguousarray(m.xyz, dtype=np.float64)
    conn = np.ascontiguousarray(m.conn, dtype=np.int32)
    path = tmp_path / "mesh.bin"
    assert abi.beta_gpu_write_mesh(str(path).encode(), 1, 3, m.nnode, xyz.ctypes.data, m.nelem, 8,
                                   conn.ctypes.data, 1) == 0
    nums = np.arange(1, m.nnode + 1, dtype=np.int32)
    nb, xb = r.node_records(nums, xyz, tmp_path / "nodes.bin")
    np.testing.assert_array_equal(nb, nums)
    np.testing.assert_array_equal(xb, xyz)
    ours = path.read_bytes()[12:12 + 28 * m.nnode]  # after the three-int header
    assert ours == (tmp_path / "nodes.bin").read_bytes()


def test_geometric_nonlinear_element_equals_the_reference(oracle):
    """ElasticityElement3D with analysisType GEOMETRIC_NONLINEAR (the element of
    BasicModel::iterate): B with the displacement-gradient terms, Green-Lagrange
    strain, the initial-stress term (ElasticityElement3D.cpp:84-160, 560-641).
    The oracle's tangent and internal force equal the reference's own code's
    on distorted elements at large displacements (golden, and live where
    oracle/_ref is built)."""
    g = _load("ref_gnl.json")
    live = oracle.RefLeaf() if oracle.RefLeaf.available() else None
    for case in g["cases"]:
        X, C6, u = np.array(case["X"]), oracle.cmat_ortho3d(case["m9"]), np.array(case["u"])
        for order in (2, 3):
            K, F = oracle.gnl_hex8(X, C6, u, order)
            Kr, Fr = np.array(case[str(order)]["K"]), np.array(case[str(order)]["F"])
            assert np.abs(np.triu(K) - Kr).max() <= 1e-15 * np.abs(Kr).max()
            assert np.abs(F - Fr).max() <= 1e-15 * np.abs(Fr).max()
            if live is not None:
                Kl, _, _ = live.elastic_update_gnl(X, C6, order, "K", u)
                _, Fl, _ = live.elastic_update_gnl(X, C6, order, "F", u)
                np.testing.assert_array_equal(np.triu(Kl), Kr)
                np.testing.assert_array_equal(Fl, Fr)


def test_geometric_nonlinear_tangent_is_the_derivative_of_the_force(oracle):
    """The tangent (material + initial-stress terms) is the derivative of the
    internal force: central differences agree to the step's truncation."""
    rng = np.random.default_rng(5)
    X = np.array([[0, 0, 0], [0, 1, 0], [0, 1, 1], [0, 0, 1], [1, 0, 0], [1, 1, 0], [1, 1, 1], [1, 0, 1]], float)
    X = X + 0.05 * rng.normal(size=X.shape)
    C6 = oracle.cmat_ortho3d([100, 90, 110, 0.3, 0.25, 0.28, 40, 35, 45])
    u = 0.1 * rng.normal(size=24)
    K, _ = oracle.gnl_hex8(X, C6, u)
    Kf = np.triu(K) + np.triu(K, 1).T
    h = 1e-6
    J = np.zeros((24, 24))
    for j in range(24):
        e = np.zeros(24)
        e[j] = h
        J[:, j] = (oracle.gnl_hex8(X, C6, u + e)[1] - oracle.gnl_hex8(X, C6, u - e)[1]) / (2 * h)
    assert np.abs(J - Kf).max() <= 1e-8 * np.abs(Kf).max()
    K0, F0 = oracle.gnl_hex8(X, C6, np.zeros(24))
    _, KL = oracle.ke_hex8(X, C6)
    np.testing.assert_allclose(np.triu(K0), np.triu(KL), rtol=0, atol=1e-13 * np.abs(KL).max())
    assert np.abs(F0).max() == 0.0


def test_newton_converges_quadratically_on_a_cantilever(oracle):
    """BasicModel::iterate restated: from zero the first step is the linear
    solution; the loop stops once max |R| < 1e-10, the last steps square the
    residual, and a load 1000x smaller gives the linear answer."""
    m = W.cantilever_hex8(nx=12, ny=2, nz=2, load=6.0)
    s = oracle.System(m)
    s.set_bc(m.restrained, m.prescribed, m.load)
    s.build_pattern()
    rc, u, hist, its, lin = s.newton(m.params, m.order, np.zeros(m.ndof), max_residual=1e-10, max_newton=40,
                                     eps=1e-13)
    assert rc == 0 and hist[-1] < 1e-10 and 3 <= its <= 20
    assert hist[-2] < 1e-3 and hist[-1] < 10 * hist[-2] ** 1.5
    ms = W.cantilever_hex8(nx=12, ny=2, nz=2, load=6e-3)
    s2 = oracle.System(ms)
    s2.set_bc(ms.restrained, ms.prescribed, ms.load)
    s2.build_pattern()
    rc, u2, _, _, _ = s2.newton(ms.params, ms.order, np.zeros(ms.ndof), max_residual=1e-14, max_newton=40, eps=1e-14)
    s3 = oracle.System(ms)
    s3.set_bc(ms.restrained, ms.prescribed, ms.load)
    s3.build_pattern()
    s3.assemble(ms.params, ms.order)
    _, ulin, _ = s3.solve(eps=1e-14, maxit=100000)
    assert np.linalg.norm(u2 - ulin) <= 2e-3 * np.linalg.norm(ulin)
    tip = np.isclose(m.xyz[:, 0], m.meta["length"])
    assert u[3 * np.nonzero(tip)[0] + 2].mean() > 1e3 * u2[3 * np.nonzero(tip)[0] + 2].mean()  # both negative
