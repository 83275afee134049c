"""Seeded synthetic models for the assembly + PCG path.

Every generator returns a :class:`Model`: a structured mesh in BETA's local
node order (hex8: nodes 0-3 on xi=-1 with (eta,zeta) = (-,-),(+,-),(+,+),
(-,+), nodes 4-7 the same on xi=+1; quad4 counter-clockwise), the node-major
interleaved dof numbering of Node::setNumDofPerNode (first_dof = ndpn*node),
per-element material parameters in the element kind's parameter order, and
restraints / prescribed values / nodal loads as BETA's DisplacementLoad /
PlaneDisplacement / PointLoad would produce them.  Tractions and pressures
enter as consistent nodal loads, the way BETA applies them with PointLoad.

Random values come from a counter-based generator (splitmix64 of
seed/stream/index, Box-Muller for normals), so a value depends only on
(seed, stream, element id) and every consumer sees the same inputs.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import _abi

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _splitmix64(x: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        return _splitmix64_raw(np.asarray(x, dtype=np.uint64))


def _splitmix64_raw(x: np.ndarray) -> np.ndarray:
    x = (x + np.uint64(0x9E3779B97F4A7C15)) & _M64
    z = x
    z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & _M64
    z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & _M64
    return z ^ (z >> np.uint64(31))


def uniform(seed: int, stream: int, idx) -> np.ndarray:
    """U[0,1) keyed by (seed, stream, idx)."""
    idx = np.asarray(idx, dtype=np.uint64)
    key = _splitmix64(np.uint64(seed) * np.uint64(0x100000001B3) + np.uint64(stream) * np.uint64(0x9E3779B1))
    with np.errstate(over="ignore"):
        u = _splitmix64(idx ^ key)
    return (u >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def normal(seed: int, stream: int, idx) -> np.ndarray:
    u1 = uniform(seed, 2 * stream, idx)
    u2 = uniform(seed, 2 * stream + 1, idx)
    return np.sqrt(-2.0 * np.log1p(-u1)) * np.cos(2.0 * math.pi * u2)


@dataclasses.dataclass
class Model:
    name: str
    kind: int
    ndim: int
    xyz: np.ndarray          # (nnode, ndim) float64
    conn: np.ndarray         # (nelem, nnpe) int32, BETA local order
    ndpn: int
    params: np.ndarray       # (nelem, nparams) float64
    restrained: np.ndarray   # (ndof,) uint8
    prescribed: np.ndarray   # (ndof,) float64
    load: np.ndarray         # (ndof,) float64
    order: int
    meta: dict = dataclasses.field(default_factory=dict)

    @property
    def nnode(self):
        return self.xyz.shape[0]

    @property
    def nelem(self):
        return self.conn.shape[0]

    @property
    def nnpe(self):
        return self.conn.shape[1]

    @property
    def ndof(self):
        return self.nnode * self.ndpn

    @property
    def first_dof(self):
        return (np.arange(self.nnode, dtype=np.int32) * self.ndpn).astype(np.int32)

    def nbytes_inputs(self):
        return sum(a.nbytes for a in (self.xyz, self.conn, self.params, self.restrained, self.prescribed,
                                      self.load)) + self.first_dof.nbytes


# ---------------------------------------------------------------------------
def grid_quad4(nx, ny, lx=1.0, ly=1.0):
    xs = np.linspace(0.0, lx, nx + 1)
    ys = np.linspace(0.0, ly, ny + 1)
    X, Y = np.meshgrid(xs, ys, indexing="xy")  # node id = i + (nx+1)*j
    xyz = np.stack([X.ravel(), Y.ravel()], axis=1)
    i, j = np.meshgrid(np.arange(nx), np.arange(ny), indexing="xy")
    i, j = i.ravel(), j.ravel()
    nid = lambda a, b: a + (nx + 1) * b  # noqa: E731
    conn = np.stack([nid(i, j), nid(i + 1, j), nid(i + 1, j + 1), nid(i, j + 1)], axis=1).astype(np.int32)
    return xyz, conn


def grid_hex8(nx, ny, nz, lx=1.0, ly=1.0, lz=1.0):
    xs = np.linspace(0.0, lx, nx + 1)
    ys = np.linspace(0.0, ly, ny + 1)
    zs = np.linspace(0.0, lz, nz + 1)
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")  # node id = i + (nx+1)*(j + (ny+1)*k)
    xyz = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()

    def nid(a, b, c):
        return a + (nx + 1) * (b + (ny + 1) * c)

    # BETA hex8 order: xi ~ x, eta ~ y, zeta ~ z
    conn = np.stack([
        nid(i, j, k), nid(i, j + 1, k), nid(i, j + 1, k + 1), nid(i, j, k + 1),
        nid(i + 1, j, k), nid(i + 1, j + 1, k), nid(i + 1, j + 1, k + 1), nid(i + 1, j, k + 1),
    ], axis=1).astype(np.int32)
    return xyz, conn


def iso3d_params(E, nu):
    E = np.asarray(E, dtype=np.float64)
    nu = np.broadcast_to(np.asarray(nu, dtype=np.float64), E.shape)
    G = E / (2.0 * (1.0 + nu))
    return np.stack([E, E, E, nu, nu, nu, G, G, G], axis=1)


def pstress_params(E, nu):
    E = np.asarray(E, dtype=np.float64)
    nu = np.broadcast_to(np.asarray(nu, dtype=np.float64), E.shape)
    return np.stack([E, E, nu, E / (2.0 * (1.0 + nu))], axis=1)


# ---- configuration 1: quad4 plane stress plate ------------------------------
def plate_quad4(n=64, E=70e3, nu=0.3, traction=1.0, order=2):
    """Unit square, n x n quad4, left edge clamped, +x traction on the right edge."""
    xyz, conn = grid_quad4(n, n)
    nnode = xyz.shape[0]
    ndof = 2 * nnode
    rest = np.zeros(ndof, np.uint8)
    left = np.where(np.isclose(xyz[:, 0], 0.0))[0]
    rest[2 * left] = 1
    rest[2 * left + 1] = 1
    load = np.zeros(ndof)
    right = np.where(np.isclose(xyz[:, 0], 1.0))[0]
    h = 1.0 / n
    w = np.full(right.shape, traction * h)
    w[np.isclose(xyz[right, 1], 0.0) | np.isclose(xyz[right, 1], 1.0)] = traction * h / 2
    load[2 * right] = w
    params = pstress_params(np.full(conn.shape[0], E), nu)
    return Model(f"quad4_plate_{n}", _abi.QUAD4_PSTRESS, 2, xyz, conn, 2, params, rest, np.zeros(ndof), load,
                 order, {"n": n})


# ---- configuration 2: hex8 cube, lognormal moduli ---------------------------
def cube_hex8(n=100, seed=2024, pressure=1.0, order=2, sigma=0.5, nu_lo=0.20, nu_hi=0.35):
    """[0,1]^3, n^3 hex8; E_e = 1e4 exp(N(0, sigma^2)), nu_e ~ U[nu_lo, nu_hi];
    z=0 clamped; pressure p on z=1 as -z nodal loads p*A/4 per face corner."""
    xyz, conn = grid_hex8(n, n, n)
    nnode = xyz.shape[0]
    ne = conn.shape[0]
    eid = np.arange(ne, dtype=np.uint64)
    E = 1e4 * np.exp(sigma * normal(seed, 1, eid))
    nu = nu_lo + (nu_hi - nu_lo) * uniform(seed, 3, eid)
    params = iso3d_params(E, nu)
    ndof = 3 * nnode
    rest = np.zeros(ndof, np.uint8)
    bot = np.where(np.isclose(xyz[:, 2], 0.0))[0]
    for c in range(3):
        rest[3 * bot + c] = 1
    top = np.where(np.isclose(xyz[:, 2], 1.0))[0]
    h = 1.0 / n
    onx = np.isclose(xyz[top, 0], 0.0) | np.isclose(xyz[top, 0], 1.0)
    ony = np.isclose(xyz[top, 1], 0.0) | np.isclose(xyz[top, 1], 1.0)
    nface = 4 // (1 + onx.astype(int)) // (1 + ony.astype(int))
    load = np.zeros(ndof)
    load[3 * top + 2] = -pressure * h * h / 4.0 * nface
    return Model(f"hex8_cube_{n}", _abi.HEX8_ELASTIC, 3, xyz, conn, 3, params, rest, np.zeros(ndof), load, order,
                 {"n": n, "seed": seed})


# ---- configuration 3: transient diffusion slab ------------------------------
def heat_slab(nx=256, ny=256, nz=64, seed=7, order=3, lx=1.0, ly=1.0):
    """[0,lx]x[0,ly]x[0,lz] with lz = lx*nz/nx (cubic cells); k_e = exp(N(0,1)),
    capacity 1; T = 0 on all faces; u0 a Gaussian bump (sigma = 0.1 lx)
    at the centre, zeroed on the Dirichlet nodes."""
    lz = lx * nz / nx
    xyz, conn = grid_hex8(nx, ny, nz, lx, ly, lz)
    nnode = xyz.shape[0]
    ne = conn.shape[0]
    k = np.exp(normal(seed, 5, np.arange(ne, dtype=np.uint64)))
    params = np.stack([k, k, k, np.ones(ne)], axis=1)
    on = (np.isclose(xyz[:, 0], 0) | np.isclose(xyz[:, 0], lx) | np.isclose(xyz[:, 1], 0) |
          np.isclose(xyz[:, 1], ly) | np.isclose(xyz[:, 2], 0) | np.isclose(xyz[:, 2], lz))
    rest = on.astype(np.uint8)
    sig = 0.1 * lx
    c = np.array([lx / 2, ly / 2, lz / 2])
    u0 = np.exp(-np.sum((xyz - c) ** 2, axis=1) / (2 * sig * sig))
    u0[on] = 0.0
    m = Model(f"heat_slab_{nx}x{ny}x{nz}", _abi.HEX8_HEAT, 3, xyz, conn, 1, params, rest, np.zeros(nnode),
              np.zeros(nnode), order, {"nx": nx, "ny": ny, "nz": nz, "seed": seed})
    m.meta["u0"] = u0
    return m


# ---- configuration 4: two-phase RVE cubes ------------------------------------
def rve_hex8(n, seed, order=2, E_matrix=1e3, contrast=10.0, nu=0.3, ux=0.01):
    """n^3 hex8 unit cube with non-overlapping spherical inclusions placed by
    seeded rejection until the drawn volume fraction ~U[0.2,0.4] is reached
    (radii ~U[0.05,0.15]); E_incl = contrast*E_matrix; x=0 clamped, u_x = ux on x=1."""
    xyz, conn = grid_hex8(n, n, n)
    ne = conn.shape[0]
    vf_target = 0.2 + 0.2 * uniform(seed, 11, 0)[()]
    tries = np.arange(20000, dtype=np.uint64)
    R = 0.05 + 0.10 * uniform(seed, 12, tries)
    CC = np.stack([uniform(seed, 13, tries), uniform(seed, 14, tries), uniform(seed, 15, tries)], axis=1)
    CC = R[:, None] + (1 - 2 * R[:, None]) * CC
    acc_c = np.zeros((0, 3))
    acc_r = np.zeros(0)
    vol = 0.0
    for t in range(len(R)):
        if vol >= vf_target:
            break
        if acc_r.size and np.any(np.sqrt(((acc_c - CC[t]) ** 2).sum(axis=1)) < R[t] + acc_r):
            continue
        acc_c = np.vstack([acc_c, CC[t]])
        acc_r = np.append(acc_r, R[t])
        vol += 4.0 / 3.0 * math.pi * R[t] ** 3
    centres, radii = list(acc_c), list(acc_r)
    cen = xyz[conn].mean(axis=1)
    inc = np.zeros(ne, bool)
    for cc, r in zip(centres, radii):
        inc |= np.sum((cen - cc) ** 2, axis=1) <= r * r
    E = np.where(inc, contrast * E_matrix, E_matrix)
    params = iso3d_params(E, nu)
    ndof = 3 * xyz.shape[0]
    rest = np.zeros(ndof, np.uint8)
    presc = np.zeros(ndof)
    x0 = np.where(np.isclose(xyz[:, 0], 0.0))[0]
    x1 = np.where(np.isclose(xyz[:, 0], 1.0))[0]
    for c in range(3):
        rest[3 * x0 + c] = 1
    rest[3 * x1] = 1
    presc[3 * x1] = ux
    return Model(f"rve_{n}_{seed}", _abi.HEX8_ELASTIC, 3, xyz, conn, 3, params, rest, presc, np.zeros(ndof), order,
                 {"n": n, "seed": seed, "vf": float(inc.mean()), "ninc": len(radii)})


def rve_batch(count=512, seed=99, n_lo=8, n_hi=40):
    sides = n_lo + (uniform(seed, 21, np.arange(count, dtype=np.uint64)) * (n_hi - n_lo + 1)).astype(int)
    sides = np.minimum(sides, n_hi)
    return [rve_hex8(int(n), seed * 100003 + i) for i, n in enumerate(sides)]
