"""Generates tests/golden/*.json.

Run from the repository root, in a checkout that has the reference tree and
the compiled reference leaf library (``make -C oracle``):

    python tests/golden/gen_golden.py

* ``ref_quadrature.json`` -- Gauss-Legendre points/weights (orders 1-8) and the
  hex/quad tensor lists (orders 1-4) produced by the reference's own
  beta/math/gaussQuadrature/gauss.cpp, and hex8/quad4 shape functions and
  local derivatives (plus the quad8/tri6 surface shapes SurfaceLoad uses)
  from beta/elements/shape.cpp, at a fixed set of points, and the
  conductivity matrix of one distorted quad4 accumulated by the reference's
  own HeatTransferElement2Dtransient::addToKe over its own Gauss points; for
  one distorted hex8, the 3D element's addToKe (anisotropic k) and addToMe
  and the step terms formK_s / formF_s_new; for a distorted hex8 and quad4,
  the elasticity elements' stiffness (calculateBmatrix + addToKe) and, for
  the hex8, the internal force (derivativesOfFields + calculateStrain +
  addToFe) for a general constitutive matrix; the element driver
  update("KF") and getVolAvgValues of both elasticity elements, and the
  diffusion elements' driver update("KM").
  These are outputs of the reference code itself (oracle/_ref).
* ``ref_gnl.json`` -- the reference's own ElasticityElement3D with
  analysisType GEOMETRIC_NONLINEAR (the element of BasicModel::iterate):
  tangent and internal force of distorted hex8 elements at given
  displacements (``python tests/golden/gen_golden.py gnl`` writes this file
  alone).
* ``ref_cg.json`` -- the reference's own Jacobi-PCG (sparse.cpp
  SymmetricSparseMatrix::solve, compiled unmodified with largeMatrix.cpp)
  on small assembled systems read by its own readMatrixAddressFormat from
  files in the lower-triangle address format: iterations and solutions.
* ``ref_exchange.json`` -- SHA-256 of the files the reference's own
  writers (sparse.cpp printMatrixAddressFormat[Upper], printCompressedRowFormat;
  SparseMatrixUtility.cpp writeCSRMatrixIn{ASCII,Binary}) produce for the
  assembled lower triangle of a small RVE.
* ``ref_materials.json`` -- constitutive matrices built by the reference's
  own material code (beta/materials/3D/elastic.cpp ElasticMaterial::read of
  a readModuli block, beta/materials/2D/pStress.cpp PlaneStress::read,
  beta_ext/diffusion/material/heatTransferMaterial.cpp readConductivity and
  calculateFlux) and
  inverses by its own Matrix::invert (beta/math/matrix.cpp), compiled
  unmodified into oracle/_ref/libbeta_ref_material.so.
* ``ref_equations.json`` -- the reference's own global assembly
  (beta/math/equation/equation.cpp Equations: setRestraint, setupStorage,
  setSolution, specifyNonZeroLocation, allocate, zeroMatrix, addMatrix,
  addLoadToEqn, solve; with addeqn.cpp, sparse.cpp, largeMatrix.cpp and
  matrix.cpp, compiled unmodified into oracle/_ref/libbeta_ref_equations.so)
  on small meshes -- renumbered, with nonzero prescribed values, an unused
  node -- given the oracle's element matrices: the lower triangle (CSR), the
  pseudo-load vector and the solution; and a solve whose unused free node
  leaves zero-diagonal rows, with the ReplaceZeroDiagonal option set.
* ``ref_heat_steps.json`` -- backward-Euler steps of a small hex8 slab
  (with and without a heat input) and a quad4 plate with a heat input
  (the 2D element), alpha 1 and 0.5, composed from the
  reference's own code in DiffusionModel's order (DiffusionModel.cpp:743-818,
  322-347): per element its formK_s / formF_s_new
  (HeatTransferElement3DTransient.cpp) on the oracle's element K and M, the
  Equations addMatrix of Mbar_e with Fbar_e, and solve from u_s.
* ``ref_internal_force.json`` -- the global internal force of a renumbered
  hex8 cube under a random displacement: element forces from the
  reference's ElasticityElement3D (derivativesOfFields, calculateStrain,
  addToFe) summed by its Equations::assembleResultantVector with the
  restraint mask.
* ``ref_matrix_kat.json`` -- the known answers written in the reference's
  DEBUG_MATRIX_CLASS main (beta/math/matrix.cpp:679-696).
* ``oracle_small.json`` -- small end-to-end cases from the oracle (element
  matrices, assembled lower-triangle systems, PCG solutions) used as
  regression fixtures by the GPU parity tests.
"""
import dataclasses
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import beta_oracle as bo  # noqa: E402
from betanoox_b200 import workloads as W  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
SAMPLE_HEX = [(-0.9, 0.1, 0.7), (0.3, -0.7, 0.1), (-0.57735, 0.57735, -0.57735), (0.0, 0.0, 0.0), (1.0, -1.0, 1.0)]
SAMPLE_QUAD = [(-0.9, 0.1), (0.3, -0.7), (0.57735, -0.57735), (0.0, 0.0), (-1.0, 1.0)]
SAMPLE_TRI = [(0.1, 0.2), (1.0 / 3, 1.0 / 3), (0.7, 0.05), (0.0, 0.0), (0.5, 0.5)]


def ref_quadrature():
    r = bo.RefLeaf()
    out = {"gauss": {}, "hex": {}, "quad": {}, "shape_hex8": [], "shape_quad4": [], "shape_quad8": [],
           "shape_tri6": []}
    for k in range(1, 9):
        x, w = r.gauss_1d(k)
        out["gauss"][str(k)] = {"x": x.tolist(), "w": w.tolist()}
    for o in range(1, 5):
        a = r.hex_points(o)
        out["hex"][str(o)] = {"xi": a[0].tolist(), "eta": a[1].tolist(), "zeta": a[2].tolist(), "w": a[3].tolist()}
        b = r.quad_points(o)
        out["quad"][str(o)] = {"xi": b[0].tolist(), "eta": b[1].tolist(), "w": b[2].tolist()}
    for p in SAMPLE_HEX:
        S, d0, d1, d2 = r.shape_hex8(*p)
        out["shape_hex8"].append({"at": p, "S": S.tolist(), "dxi": d0.tolist(), "deta": d1.tolist(), "dzeta": d2.tolist()})
    for p in SAMPLE_QUAD:
        S, d0, d1 = r.shape_quad4(*p)
        out["shape_quad4"].append({"at": p, "S": S.tolist(), "dxi": d0.tolist(), "deta": d1.tolist()})
        S, d0, d1 = r.shape_quad8(*p)
        out["shape_quad8"].append({"at": p, "S": S.tolist(), "dxi": d0.tolist(), "deta": d1.tolist()})
    for p in SAMPLE_TRI:
        S, d0, d1 = r.shape_tri6(*p)
        out["shape_tri6"].append({"at": p, "S": S.tolist(), "dxi": d0.tolist(), "deta": d1.tolist()})
    xy = np.array([[0.0, 0.0], [1.3, 0.1], [1.1, 0.9], [-0.1, 1.2]])
    out["heat2d_ke"] = {"xy": xy.tolist(), "k11": 2.0, "k22": 0.7, "orders": {}}
    for order in (2, 3):
        xi, eta, w = r.quad_points(order)
        K = np.zeros((4, 4))
        for a, b, wt in zip(xi, eta, w):
            _, dxi, deta = r.shape_quad4(a, b)
            J = np.array([dxi @ xy, deta @ xy])
            g = np.linalg.solve(J, np.array([dxi, deta]))
            K = r.heat2d_add_to_ke(2.0, 0.7, 0.0, g[0], g[1], np.linalg.det(J) * wt, K)
        out["heat2d_ke"]["orders"][str(order)] = K.tolist()
    # 3D diffusion element: addToKe (full anisotropic k) + addToMe over the
    # reference's hex Gauss points, then formK_s / formF_s_new of one step
    X = (np.array([[0, 0, 0], [0, 1, 0], [0, 1, 1], [0, 0, 1], [1, 0, 0], [1, 1, 0], [1, 1, 1], [1, 0, 1]], float)
         * np.array([1.2, 0.9, 1.1]) + np.random.default_rng(2).uniform(-0.08, 0.08, (8, 3)))
    k9 = np.array([[2.0, 0.3, 0.1], [0.3, 1.5, 0.2], [0.1, 0.2, 0.8]])
    us = np.random.default_rng(5).normal(size=8)
    h3 = {"xyz": X.tolist(), "k9": k9.tolist(), "cap": 1.7, "u_s": us.tolist(), "a1": 1.0, "a2": 0.0,
          "dt": 1e-3, "orders": {}}
    for order in (2, 3):
        xi, eta, zeta, w = r.hex_points(order)
        K, M = np.zeros((8, 8)), np.zeros((8, 8))
        for a, b, c, wt in zip(xi, eta, zeta, w):
            S, d0, d1, d2 = r.shape_hex8(a, b, c)
            J = np.array([d0 @ X, d1 @ X, d2 @ X])
            g = np.linalg.solve(J, np.array([d0, d1, d2]))
            K, M = r.heat3d_add_to_km(k9, 1.7, S, g[0], g[1], g[2], np.linalg.det(J) * wt, K, M)
        Mb, F = r.heat3d_step_terms(K, M, us, 1.0, 0.0, 1e-3)
        h3["orders"][str(order)] = {"K": K.tolist(), "M": M.tolist(), "Mbar": Mb.tolist(), "F": F.tolist()}
    out["heat3d"] = h3
    # elasticity elements: ElasticityElement3D's calculateBmatrix + addToKe and
    # derivativesOfFields + calculateStrain + addToFe (hex8, general SPD 6x6 C),
    # ElasticityElement2D's (quad4, general SPD 3x3 C), over the reference's
    # Gauss points
    rng = np.random.default_rng(7)
    X = (np.array([[0, 0, 0], [0, 1, 0], [0, 1, 1], [0, 0, 1], [1, 0, 0], [1, 1, 0], [1, 1, 1], [1, 0, 1]], float)
         * np.array([1.1, 0.95, 1.05]) + rng.uniform(-0.08, 0.08, (8, 3)))
    A = rng.normal(size=(6, 6))
    C6 = A @ A.T + 6 * np.eye(6)
    u = rng.normal(size=24)
    e3 = {"xyz": X.tolist(), "C": C6.tolist(), "u": u.tolist(), "orders": {}}
    for order in (2, 3):
        xi, eta, zeta, w = r.hex_points(order)
        K, F = np.zeros((24, 24)), np.zeros(24)
        for a, b, c, wt in zip(xi, eta, zeta, w):
            S, d0, d1, d2 = r.shape_hex8(a, b, c)
            J = np.array([d0 @ X, d1 @ X, d2 @ X])
            g = np.linalg.solve(J, np.array([d0, d1, d2]))
            K, F, _ = r.elastic_point(C6, g[0], g[1], g[2], np.linalg.det(J) * wt, K, u=u, Fe=F)
        e3["orders"][str(order)] = {"K": K.tolist(), "F": F.tolist()}
    out["elastic3d"] = e3
    X2 = np.array([[0.0, 0.0], [1.2, 0.1], [1.1, 0.9], [-0.05, 1.0]])
    A = rng.normal(size=(3, 3))
    C3 = A @ A.T + 3 * np.eye(3)
    e2 = {"xy": X2.tolist(), "C": C3.tolist(), "orders": {}}
    for order in (2, 3):
        xi, eta, w = r.quad_points(order)
        K = np.zeros((8, 8))
        for a, b, wt in zip(xi, eta, w):
            S, d0, d1 = r.shape_quad4(a, b)
            J = np.array([d0 @ X2, d1 @ X2])
            g = np.linalg.solve(J, np.array([d0, d1]))
            K, _, _ = r.elastic_point(C3, g[0], g[1], None, np.linalg.det(J) * wt, K)
        e2["orders"][str(order)] = {"K": K.tolist()}
    out["elastic2d"] = e2
    out["elastic_driver"] = elastic_driver_case(r)
    out["heat_driver"] = heat_driver_case(r)
    out["source"] = ("reference gauss.cpp + shape.cpp + HeatTransfer{2D,3D}Transient and Elasticity{2D,3D} "
                     "element files compiled unmodified (oracle/_ref)")
    return out


def heat_driver_inputs():
    rng = np.random.default_rng(41)
    X = (np.array([[0, 0, 0], [0, 1, 0], [0, 1, 1], [0, 0, 1], [1, 0, 0], [1, 1, 0], [1, 1, 1], [1, 0, 1]], float)
         * np.array([1.2, 0.9, 1.1]) + rng.uniform(-0.08, 0.08, (8, 3)))
    X2 = np.array([[0.0, 0.0], [1.2, 0.1], [1.1, 0.9], [-0.05, 1.0]])
    return X, [2.0, 1.5, 0.8], 1.7, X2, [2.0, 1.5], 1.3


def heat_driver_case(r):
    """The reference's diffusion element driver update("KM") on one hex8 and
    one quad4 (the 2D element through the 3D element's driver)."""
    X, k3, c3, X2, k2, c2 = heat_driver_inputs()
    out = {"hex8": {}, "quad4": {}}
    for order in (2, 3):
        K, M = r.heat_update(X, k3, c3, order)
        out["hex8"][str(order)] = {"K": K.tolist(), "M": M.tolist()}
        K, M = r.heat_update(X2, k2, c2, order)
        out["quad4"][str(order)] = {"K": K.tolist(), "M": M.tolist()}
    return out


def elastic_driver_inputs():
    rng = np.random.default_rng(31)
    X = (np.array([[0, 0, 0], [0, 1, 0], [0, 1, 1], [0, 0, 1], [1, 0, 0], [1, 1, 0], [1, 1, 1], [1, 0, 1]], float)
         * np.array([1.2, 0.9, 1.1]) + rng.uniform(-0.08, 0.08, (8, 3)))
    m9 = [150.0, 12.0, 9.0, 0.25, 0.32, 0.28, 5.0, 3.5, 4.2]
    u = rng.normal(size=24)
    X2 = np.array([[0.0, 0.0], [1.2, 0.1], [1.1, 0.9], [-0.05, 1.0]])
    m4 = [140.0, 10.0, 0.3, 5.0]
    u2 = rng.normal(size=8)
    return X, m9, u, X2, m4, u2


def elastic_driver_case(r):
    """The reference's element driver update("KF") and getVolAvgValues on one
    hex8 and one quad4 with material constants."""
    X, m9, u, X2, m4, u2 = elastic_driver_inputs()
    C6, C3 = bo.cmat_ortho3d(m9), bo.cmat_plane_stress(m4)
    out = {"hex8": {}, "quad4": {}}
    for order in (2, 3):
        K, F, sums = r.elastic_update(X, C6, order, "KF", u)
        out["hex8"][str(order)] = {"K": K.tolist(), "F": F.tolist(), "vol_avg": r.elastic_vol_avg(X, C6, order, u).tolist()}
    K, F, sums = r.elastic_update(X2, C3, 2, "K")
    va = r.elastic_vol_avg(X2, C3, 2, u2)
    # the plane element's getVolAvgValues fills 3 stress / strain components
    out["quad4"]["2"] = {"K": K.tolist(), "volume": float(va[0]), "stress": va[1:4].tolist(), "strain": va[7:10].tolist()}
    return out


def gnl_inputs():
    """Distorted hex8 elements with general orthotropic constants and
    displacements large enough for the nonlinear terms to matter."""
    rng = np.random.default_rng(47)
    cases = []
    for k in range(3):
        X = (np.array([[0, 0, 0], [0, 1, 0], [0, 1, 1], [0, 0, 1], [1, 0, 0], [1, 1, 0], [1, 1, 1], [1, 0, 1]], float)
             * np.array([1.3, 0.8, 1.0]) + rng.uniform(-0.07, 0.07, (8, 3)))
        m9 = [100.0 + 20 * k, 80.0, 120.0, 0.28, 0.31, 0.25, 30.0, 40.0, 35.0]
        u = 0.1 * rng.normal(size=24)
        cases.append((X, m9, u))
    return cases


def ref_gnl():
    """The reference's own ElasticityElement3D with analysisType
    GEOMETRIC_NONLINEAR (update "K" and "F" at displacements u): tangent
    (upper triangle) and internal force, orders 2 and 3."""
    r = bo.RefLeaf()
    out = {"source": "reference ElasticityElement3D.cpp update('K'/'F') with analysisType GEOMETRIC_NONLINEAR "
                     "(oracle/_ref)", "cases": []}
    for X, m9, u in gnl_inputs():
        C6 = bo.cmat_ortho3d(m9)
        case = {"X": X.tolist(), "m9": m9, "u": u.tolist()}
        for order in (2, 3):
            K, _, _ = r.elastic_update_gnl(X, C6, order, "K", u)
            _, F, _ = r.elastic_update_gnl(X, C6, order, "F", u)
            case[str(order)] = {"K": np.triu(K).tolist(), "F": F.tolist()}
        out["cases"].append(case)
    return out


def ref_cg():
    import tempfile
    from betanoox_b200 import _abi, write_lower
    r = bo.RefLeaf()
    out = {"source": "reference sparse.cpp + largeMatrix.cpp compiled unmodified (oracle/_ref)", "cases": []}
    for name, m in [("plate_quad4_12", W.plate_quad4(12)), ("cube_hex8_5_s3", W.cube_hex8(5, seed=3)),
                    ("heat_plate_12x9", W.heat_plate(12, 9, heat=2.0))]:
        s = bo.System(m)
        s.set_bc(m.restrained, m.prescribed, m.load)
        s.build_pattern()
        s.assemble(m.params, m.order)
        rp, col, val = s.export_lower()
        b = s.rhs()
        with tempfile.TemporaryDirectory() as d:
            p = os.path.join(d, "k.txt")
            write_lower(p, _abi.FMT_ADDRESS_LOWER, rp, col, val)
            x, it = r.sparse_solve_file(p, b, 1e-10)
        out["cases"].append({"name": name, "eps": 1e-10, "iterations": it, "x": x.tolist()})
    return out


def ref_exchange():
    import hashlib
    import tempfile
    r = bo.RefLeaf()
    m = W.rve_hex8(5, 3)
    s = bo.System(m)
    s.set_bc(m.restrained, m.prescribed, m.load)
    s.build_pattern()
    s.assemble(m.params, m.order)
    rp, col, val = s.export_lower()
    out = {"source": "reference sparse.cpp / SparseMatrixUtility.cpp writers compiled unmodified (oracle/_ref)",
           "model": "rve_hex8(5, 3)", "sha256": {}}
    with tempfile.TemporaryDirectory() as d:
        for name, f in [("address_lower", lambda p: r.print_lower(p, 1, rp, col, val)),
                        ("address_upper", lambda p: r.print_lower(p, 2, rp, col, val)),
                        ("compressed_row", lambda p: r.print_lower(p, 3, rp, col, val)),
                        ("csr_ascii", lambda p: r.write_csr(p, 0, rp, col, val)),
                        ("csr_binary", lambda p: r.write_csr(p, 1, rp, col, val))]:
            p = os.path.join(d, name)
            f(p)
            with open(p, "rb") as fh:
                out["sha256"][name] = hashlib.sha256(fh.read()).hexdigest()
    return out


def matrix_kat():
    return {
        "source": "beta/math/matrix.cpp:679-696 (DEBUG_MATRIX_CLASS expected values)",
        "A": [[1, 2], [3, 1]], "B": [[2, 4], [7, -3]],
        "A_plus_B": [[3, 6], [10, -2]],
        "A_times_B": [[16, -2], [13, 9]],
        "B_inverse": [[0.088235, 0.11765], [0.20588, -0.058824]],
        "B_inverse_digits": 5,
    }


def oracle_small():
    out = {}
    # element matrices on a distorted hex and quad
    xyz = np.array([[0, 0, 0], [0, 1, 0], [0, 1, 1], [0, 0, 1], [1, 0, 0], [1, 1, 0], [1, 1, 1], [1, 0, 1]], float)
    xyz = xyz * np.array([0.7, 1.1, 0.9]) + 0.05 * np.sin(np.arange(24).reshape(8, 3))
    m9 = W.iso3d_params(np.array([2.0e4]), 0.27)[0]
    C = bo.cmat_ortho3d(m9)
    st, Ke = bo.ke_hex8(xyz, C, 2)
    out["ke_hex8"] = {"xyz": xyz.tolist(), "params": m9.tolist(), "order": 2, "Ke": Ke.tolist()}
    xy = np.array([[0, 0], [1.2, 0.1], [1.0, 0.9], [-0.1, 1.0]], float)
    m4 = W.pstress_params(np.array([70e3]), 0.3)[0]
    st, Kq = bo.ke_quad4(xy, bo.cmat_plane_stress(m4), 2)
    out["ke_quad4"] = {"xy": xy.tolist(), "params": m4.tolist(), "order": 2, "Ke": Kq.tolist()}
    st, Kh, Mh = bo.km_hex8_heat(xyz, [1.3, 0.8, 2.1], 1.7, 3)
    out["km_hex8_heat"] = {"xyz": xyz.tolist(), "k": [1.3, 0.8, 2.1], "c": 1.7, "order": 3, "K": Kh.tolist(),
                           "M": Mh.tolist()}
    # a small static system
    m = W.cube_hex8(3, seed=5)
    s = bo.System(m)
    s.set_bc(m.restrained, m.prescribed, m.load)
    s.build_pattern()
    s.assemble(m.params, m.order)
    rp, col, val = s.export_lower()
    rc, u, sst = s.solve(eps=1e-12, maxit=10000)
    out["cube3"] = {"rowptr": rp.tolist(), "col": col.tolist(), "val": val.tolist(), "u": u.tolist(),
                    "iterations": sst.iterations, "eps": 1e-12}
    return out



def ref_materials():
    r = bo.RefMaterial()
    rng = np.random.default_rng(21)
    ortho = [W.iso3d_params(np.array([e]), nu)[0].tolist() for e, nu in ((200.0, 0.3), (1e4, 0.25), (3.5, 0.45))]
    ortho += [[150.0, 12.0, 9.0, 0.25, 0.32, 0.28, 5.0, 3.5, 4.2], [72.0, 72.0, 10.0, 0.3, 0.35, 0.35, 27.7, 4.0, 4.0]]
    pstress = [W.pstress_params(np.array([e]), nu)[0][:4].tolist() for e, nu in ((70e3, 0.3), (1.0, 0.49))]
    pstress += [[140.0, 10.0, 0.3, 5.0]]
    inv = []
    for n in (3, 6, 9):
        A = rng.normal(size=(n, n)) + n * np.eye(n)
        inv.append({"A": A.tolist(), "inverse": r.invert(A).tolist()})
    cond = []
    for k3, grad in (([2.5, 1.5, 0.7], [0.1, -0.2, 0.3]), ([1.0, 1.0, 1.0], [3.0, 0.5, -1.25])):
        C9, flux = r.heat_conductivity(k3, grad)
        cond.append({"k3": k3, "grad": grad, "C": C9.tolist(), "flux": flux.tolist()})
    return {"source": "reference elastic.cpp + pStress.cpp + heatTransferMaterial.cpp + matrix.cpp compiled "
                      "unmodified (oracle/_ref)",
            "ortho3d": [{"m9": m, "C": r.cmat_ortho3d(m).tolist()} for m in ortho],
            "plane_stress": [{"m4": m, "C": r.cmat_plane_stress(m).tolist()} for m in pstress],
            "invert": inv, "conductivity": cond}



def element_maps(m):
    nd = m.nnpe * m.ndpn
    return (m.first_dof[m.conn][:, :, None] + np.arange(m.ndpn)[None, None, :]).reshape(m.nelem, nd)


EQUATION_CASES = {
    "plate4_renumbered": lambda: W.renumbered(W.plate_quad4(4), 1),
    "plate4_unused_node": lambda: W.renumbered(W.plate_quad4(4), 2, unused_node=True),
    "rve2_prescribed": lambda: W.rve_hex8(2, seed=1),
    "heat_plate_4x3": lambda: W.heat_plate(4, 3, heat=2.0),
}


def zero_diag_case():
    """A renumbered plate with one node no element uses, its dofs left free:
    their rows hold only a zero diagonal (ReplaceZeroDiagonal territory)."""
    m = W.renumbered(W.plate_quad4(4), 2, unused_node=True)
    r = m.restrained.copy()
    r[-m.ndpn:] = 0
    return dataclasses.replace(m, restrained=r)


def ref_equations():
    r = bo.RefEquations()
    out = {"source": "reference equation.cpp + addeqn.cpp + sparse.cpp + largeMatrix.cpp + matrix.cpp compiled "
                     "unmodified (oracle/_ref)", "eps": 1e-10, "cases": {}}
    for name, make in EQUATION_CASES.items():
        m = make()
        nd = m.nnpe * m.ndpn
        st, Ke = bo.element_matrices_threaded(m, m.params, m.order, 0, m.nelem)
        solve = not name.endswith("unused_node")  # the unused node's row is a zero diagonal
        rp, col, val, pseudo, lv, x = r.assemble(m.ndof, element_maps(m), Ke.reshape(m.nelem, nd, nd), m.restrained,
                                                 m.prescribed, m.load, solve=solve, eps=1e-10)
        out["cases"][name] = {"rowptr": rp.tolist(), "col": col.tolist(), "val": val.tolist(),
                              "pseudo": pseudo.tolist(), "load": lv.tolist(),
                              "x": None if x is None else x.tolist()}
    m = zero_diag_case()
    nd = m.nnpe * m.ndpn
    st, Ke = bo.element_matrices_threaded(m, m.params, m.order, 0, m.nelem)
    x = r.assemble(m.ndof, element_maps(m), Ke.reshape(m.nelem, nd, nd), m.restrained, m.prescribed, m.load,
                   solve=True, eps=1e-10, zero_diag=2.5)[5]
    out["zero_diag"] = {"value": 2.5, "x": x.tolist()}
    return out



def heat_step_case(with_load, quad4=False):
    if quad4:
        return W.heat_plate(7, 5, heat=2.0)  # the 2D element, a heat input on its free nodes
    m = W.heat_slab(6, 5, 4, order=3)
    if with_load:
        rng = np.random.default_rng(17)
        load = np.where(m.restrained.astype(bool), 0.0, rng.uniform(0.0, 0.5, m.ndof))
        m = dataclasses.replace(m, load=load)
    return m


def ref_heat_step(leaf, req, m, u_s, dt, alpha, eps):
    """One step of DiffusionModel's alpha family from the reference's own
    element step terms, assembly and solve (oracle element K and M)."""
    a1, a2 = alpha * dt, (1 - alpha) * dt
    maps = element_maps(m)
    nd = maps.shape[1]
    Mb, F = np.zeros((m.nelem, nd, nd)), np.zeros((m.nelem, nd))
    for e in range(m.nelem):
        if m.nnpe == 8:
            st, K, M = bo.km_hex8_heat(m.xyz[m.conn[e]], m.params[e, :3], m.params[e, 3], order=m.order)
        else:
            st, K, M = bo.km_quad4_heat(m.xyz[m.conn[e]], m.params[e, :2], m.params[e, 3], order=m.order)
        Mb[e], F[e] = leaf.heat_step_terms(np.triu(K), np.triu(M), u_s[maps[e]], a1, a2, dt)
    x = req.assemble(m.ndof, maps, Mb, m.restrained, m.prescribed, m.load, solve=True, eps=eps, maxit=100000,
                     Fe=F, x0=u_s)[5]
    return u_s + x


def ref_heat_steps():
    leaf, req = bo.RefLeaf(), bo.RefEquations()
    out = {"source": "reference HeatTransferElement3DTransient.cpp formK_s/formF_s_new + equation.cpp "
                     "addMatrix/solve compiled unmodified (oracle/_ref), in DiffusionModel's order",
           "dt": 1e-3, "eps": 1e-14, "steps": 3, "cases": {}}
    for quad4, with_load in ((False, False), (False, True), (True, True)):
        for alpha in (1.0, 0.5):
            m = heat_step_case(with_load, quad4)
            u = m.meta["u0"].copy()
            traj = []
            for _ in range(3):
                u = ref_heat_step(leaf, req, m, u, 1e-3, alpha, 1e-14)
                traj.append(u.tolist())
            out["cases"]["%s%s_alpha%g" % ("quad4_" if quad4 else "", "load" if with_load else "free", alpha)] = {
                "with_load": with_load, "quad4": quad4, "alpha": alpha, "u": traj}
    return out



def internal_force_case():
    m = W.renumbered(W.cube_hex8(4, seed=5), 3)
    u = np.random.default_rng(1).normal(size=m.ndof)
    return m, u


def ref_internal_force():
    leaf, req = bo.RefLeaf(), bo.RefEquations()
    m, u = internal_force_case()
    maps = element_maps(m)
    xi, eta, zeta, w = leaf.hex_points(m.order)
    Fe = np.zeros((m.nelem, 24))
    for e in range(m.nelem):
        X, C6 = m.xyz[m.conn[e]], bo.cmat_ortho3d(m.params[e])
        K, F = np.zeros((24, 24)), np.zeros(24)
        for a, b, c, wt in zip(xi, eta, zeta, w):
            S, d0, d1, d2 = leaf.shape_hex8(a, b, c)
            J = np.array([d0 @ X, d1 @ X, d2 @ X])
            g = np.linalg.solve(J, np.array([d0, d1, d2]))
            K, F, _ = leaf.elastic_point(C6, g[0], g[1], g[2], np.linalg.det(J) * wt, K, u=u[maps[e]], Fe=F)
        Fe[e] = F
    return {"source": "reference ElasticityElement3D addToFe + equation.cpp assembleResultantVector compiled "
                      "unmodified (oracle/_ref)", "f": req.resultant(m.ndof, maps, Fe, m.restrained).tolist()}


if __name__ == "__main__":
    if sys.argv[1:] == ["gnl"]:  # only the geometric-nonlinear element's fixture
        with open(os.path.join(OUT, "ref_gnl.json"), "w") as f:
            json.dump(ref_gnl(), f)
        sys.exit(0)
    with open(os.path.join(OUT, "ref_gnl.json"), "w") as f:
        json.dump(ref_gnl(), f)
    with open(os.path.join(OUT, "ref_quadrature.json"), "w") as f:
        json.dump(ref_quadrature(), f)
    with open(os.path.join(OUT, "ref_cg.json"), "w") as f:
        json.dump(ref_cg(), f)
    with open(os.path.join(OUT, "ref_exchange.json"), "w") as f:
        json.dump(ref_exchange(), f, indent=1)
    with open(os.path.join(OUT, "ref_materials.json"), "w") as f:
        json.dump(ref_materials(), f, indent=1)
    with open(os.path.join(OUT, "ref_equations.json"), "w") as f:
        json.dump(ref_equations(), f)
    with open(os.path.join(OUT, "ref_heat_steps.json"), "w") as f:
        json.dump(ref_heat_steps(), f)
    with open(os.path.join(OUT, "ref_internal_force.json"), "w") as f:
        json.dump(ref_internal_force(), f)
    with open(os.path.join(OUT, "ref_matrix_kat.json"), "w") as f:
        json.dump(matrix_kat(), f, indent=1)
    with open(os.path.join(OUT, "oracle_small.json"), "w") as f:
        json.dump(oracle_small(), f)
    print("wrote golden fixtures to", OUT)
