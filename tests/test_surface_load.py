"""Surface flux loads (SurfaceLoad::applyTo, beta/BCs/SurfaceLoad.cpp:16-255).

* the oracle's surface shapes equal the reference's shape.cpp (golden
  samples from oracle/_ref, and live when that library is present);
* known answers on flat faces under a uniform flux: quad4 qA/4 per node,
  quad8 -qA/12 at corners and qA/3 at mid-sides, tri6 0 at corners and qA/3
  at mid-sides;
* the C ABI equals the oracle restatement on a curved, non-uniform case, and
  a cylinder patch under a uniform flux gets q times its area in total;
* loads land on each node's first dof and add to what the vector held;
* bad input is refused.
"""
import json
import os

import numpy as np
import pytest

from betanoox_b200 import BetaGpuError, _abi, surface_flux_load

HERE = os.path.dirname(os.path.abspath(__file__))


def _golden():
    with open(os.path.join(HERE, "golden", "ref_quadrature.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("npe,key", [(4, "shape_quad4"), (8, "shape_quad8"), (6, "shape_tri6")])
def test_oracle_shapes_equal_the_reference(oracle, npe, key):
    for case in _golden()[key]:
        N, dx, de = oracle.surface_shape(npe, *case["at"])
        np.testing.assert_allclose(N, case["S"], atol=2e-15)
        np.testing.assert_allclose(dx, case["dxi"], atol=2e-15)
        np.testing.assert_allclose(de, case["deta"], atol=2e-15)
    if oracle.RefLeaf.available():
        ref = oracle.RefLeaf()
        f = {4: ref.shape_quad4, 8: ref.shape_quad8, 6: ref.shape_tri6}[npe]
        rng = np.random.default_rng(npe)
        for _ in range(20):
            xi, eta = rng.uniform(0, 0.5, 2) if npe == 6 else rng.uniform(-1, 1, 2)
            for a, b in zip(oracle.surface_shape(npe, xi, eta), f(xi, eta)):
                np.testing.assert_allclose(a, b, atol=4e-15)


def _flat_face(npe, lx=2.0, ly=0.5, z=3.0):
    if npe == 4:
        uv = [(0, 0), (1, 0), (1, 1), (0, 1)]
    elif npe == 8:
        uv = [(0, 0), (0.5, 0), (1, 0), (1, 0.5), (1, 1), (0.5, 1), (0, 1), (0, 0.5)]
    else:
        uv = [(0, 0), (0.5, 0), (1, 0), (0.5, 0.5), (0, 1), (0, 0.5)]
    xyz = np.array([[lx * u, ly * v, z] for u, v in uv])
    area = lx * ly * (0.5 if npe == 6 else 1.0)
    return xyz, area


@pytest.mark.parametrize("npe", [4, 8, 6])
def test_uniform_flux_on_a_flat_face(oracle, npe):
    xyz, area = _flat_face(npe)
    q = 1.7
    conn = np.arange(npe)[None, :]
    fd = np.arange(npe)
    got = surface_flux_load(conn, xyz, np.full(npe, q), fd, npe)
    ora = oracle.surface_flux_load(conn, xyz, np.full(npe, q), fd, npe)
    if npe == 4:
        want = np.full(4, q * area / 4)
    elif npe == 8:
        want = np.where(np.arange(8) % 2 == 0, -q * area / 12, q * area / 3)
    else:
        want = np.where(np.arange(6) % 2 == 0, 0.0, q * area / 3)
    # the 7-point triangle rule is tabulated to 12 digits (SurfaceLoad.cpp:111-139)
    tol = 1e-11 if npe == 6 else 1e-13
    np.testing.assert_allclose(got, want, rtol=tol, atol=tol * q * area)
    np.testing.assert_allclose(ora, want, rtol=tol, atol=tol * q * area)


def _cylinder_patch(npe, n=6, r=2.0, arc=1.2, h=1.5):
    """A quarter-ish cylinder surface meshed with n x n faces (quads, or each
    quad split in two triangles); returns conn, xyz and the exact area."""
    order = 2 if npe in (6, 8) else 1
    m = order * n + 1
    t = np.linspace(0.0, arc, m)
    zz = np.linspace(0.0, h, m)
    T, Z = np.meshgrid(t, zz, indexing="xy")
    xyz = np.stack([r * np.cos(T).ravel(), r * np.sin(T).ravel(), Z.ravel()], axis=1)
    nid = lambda i, j: i + m * j  # noqa: E731
    conn = []
    for j in range(n):
        for i in range(n):
            a, b = order * i, order * j
            if npe == 4:
                conn.append([nid(a, b), nid(a + 1, b), nid(a + 1, b + 1), nid(a, b + 1)])
            elif npe == 8:
                conn.append([nid(a, b), nid(a + 1, b), nid(a + 2, b), nid(a + 2, b + 1), nid(a + 2, b + 2),
                             nid(a + 1, b + 2), nid(a, b + 2), nid(a, b + 1)])
            else:
                conn.append([nid(a, b), nid(a + 1, b), nid(a + 2, b), nid(a + 1, b + 1), nid(a, b + 2),
                             nid(a, b + 1)])
                conn.append([nid(a + 2, b + 2), nid(a + 1, b + 2), nid(a, b + 2), nid(a + 1, b + 1),
                             nid(a + 2, b), nid(a + 2, b + 1)])
    return np.array(conn), xyz, r * arc * h


@pytest.mark.parametrize("npe", [4, 8, 6])
def test_curved_surface_matches_oracle_and_area(oracle, npe):
    conn, xyz, area = _cylinder_patch(npe)
    nn = xyz.shape[0]
    fd = 3 * np.arange(nn)  # three dofs per node: loads go to the first
    rng = np.random.default_rng(11)
    q = 1.0 + rng.uniform(-0.3, 0.3, nn)
    got = surface_flux_load(conn, xyz, q, fd, 3 * nn)
    ora = oracle.surface_flux_load(conn, xyz, q, fd, 3 * nn)
    assert np.abs(got - ora).max() <= 1e-13 * np.abs(ora).max()
    assert np.all(got[1::3] == 0) and np.all(got[2::3] == 0)
    total = surface_flux_load(conn, xyz, np.ones(nn), fd, 3 * nn).sum()
    tol = 2e-3 if npe == 4 else 2e-5  # bilinear faces cut the chords
    assert abs(total - area) <= tol * area


def test_loads_add_to_the_vector():
    xyz, area = _flat_face(4)
    base = np.arange(4, dtype=float)
    out = surface_flux_load(np.arange(4)[None, :], xyz, np.ones(4), np.arange(4), 4, load=base.copy())
    np.testing.assert_allclose(out - base, area / 4)


def test_bad_input_is_refused():
    xyz, _ = _flat_face(4)
    with pytest.raises(BetaGpuError) as e:
        surface_flux_load(np.array([[0, 1, 2, 7]]), xyz, np.ones(4), np.arange(4), 4)
    assert e.value.status == _abi.ERR_ARG
    with pytest.raises(BetaGpuError) as e:
        surface_flux_load(np.array([[0, 1, 2]]), xyz, np.ones(4), np.arange(4), 4)
    assert e.value.status == _abi.ERR_ARG
    q = np.ones(4)
    q[2] = np.nan
    with pytest.raises(BetaGpuError) as e:
        surface_flux_load(np.arange(4)[None, :], xyz, q, np.arange(4), 4)
    assert e.value.status == _abi.ERR_NOT_FINITE
