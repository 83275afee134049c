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
    with np.errstate(over="ignore"):  # wrap-around multiplication is intended
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


def renumbered(m, seed, unused_node=False):
    """A copy of model m with its nodes renumbered by a seeded permutation
    (connectivity, coordinates and the per-node restraints, prescribed values
    and loads follow their nodes), optionally with one node appended that no
    element uses (its dofs restrained at zero).  The system is the same up to
    the numbering, which changes the sparsity pattern's order."""
    perm = np.random.default_rng(seed).permutation(m.nnode)      # old node -> new node
    inv = np.argsort(perm)                                        # new node -> old node
    def per_node(a, fill):
        a = np.asarray(a).reshape(m.nnode, m.ndpn)[inv]
        if unused_node:
            a = np.vstack([a, np.full((1, m.ndpn), fill, dtype=a.dtype)])
        return np.ascontiguousarray(a.reshape(-1))
    xyz = m.xyz[inv]
    if unused_node:
        xyz = np.vstack([xyz, xyz.max(axis=0) + 1.0])
    return dataclasses.replace(
        m, name=m.name + "_renumbered", xyz=np.ascontiguousarray(xyz),
        conn=np.ascontiguousarray(perm[m.conn].astype(np.int32)),
        restrained=per_node(m.restrained, 1), prescribed=per_node(m.prescribed, 0.0),
        load=per_node(m.load, 0.0), meta=dict(m.meta))


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


# ---- a cantilever for the geometric-nonlinear Newton loop --------------------
def cantilever_hex8(nx=20, ny=2, nz=2, length=10.0, width=1.0, height=1.0, load=6.0, E=1e4, nu=0.3, order=2):
    """A beam [0,length] x [0,width] x [0,height], nx x ny x nz hex8, clamped at
    x = 0, a total transverse load `load` in -z shared equally by the nodes of
    the end face x = length; isotropic E, nu.  At the default load the linear
    tip deflection is about a quarter of the length, so the deflected shape
    rotates by tens of degrees and the geometric-nonlinear solution departs
    from the linear one."""
    xyz, conn = grid_hex8(nx, ny, nz, length, width, height)
    nnode = xyz.shape[0]
    ne = conn.shape[0]
    params = iso3d_params(np.full(ne, float(E)), np.full(ne, float(nu)))
    ndof = 3 * nnode
    rest = np.zeros(ndof, np.uint8)
    root = np.where(np.isclose(xyz[:, 0], 0.0))[0]
    for c in range(3):
        rest[3 * root + c] = 1
    tip = np.where(np.isclose(xyz[:, 0], length))[0]
    f = np.zeros(ndof)
    f[3 * tip + 2] = -load / len(tip)
    return Model(f"hex8_cantilever_{nx}x{ny}x{nz}", _abi.HEX8_ELASTIC, 3, xyz, conn, 3, params, rest, np.zeros(ndof),
                 f, order, {"load": load, "length": length})


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


def heat_plate(nx=64, ny=48, seed=7, order=3, lx=1.0, heat=0.0):
    """2D transient diffusion on [0,lx]x[0,ly] (ly = lx*ny/nx, square cells),
    quad4 diffusion elements; k_e = exp(N(0,1)) in both directions, capacity 1;
    T = 0 on x = 0 and x = lx; u0 a Gaussian bump (sigma = 0.15 lx) at the
    centre, zeroed on the Dirichlet nodes; `heat` > 0 adds a uniform nodal
    heat input of heat * cell area on the free nodes."""
    ly = lx * ny / nx
    xyz, conn = grid_quad4(nx, ny, lx, ly)
    nnode = xyz.shape[0]
    ne = conn.shape[0]
    k = np.exp(normal(seed, 6, np.arange(ne, dtype=np.uint64)))
    params = np.stack([k, k, k, np.ones(ne)], axis=1)
    on = np.isclose(xyz[:, 0], 0) | np.isclose(xyz[:, 0], lx)
    rest = on.astype(np.uint8)
    sig = 0.15 * lx
    c = np.array([lx / 2, ly / 2])
    u0 = np.exp(-np.sum((xyz - c) ** 2, axis=1) / (2 * sig * sig))
    u0[on] = 0.0
    load = np.where(on, 0.0, heat * (lx / nx) ** 2)
    m = Model(f"heat_plate_{nx}x{ny}", _abi.QUAD4_HEAT, 2, xyz, conn, 1, params, rest, np.zeros(nnode), load,
              order, {"nx": nx, "ny": ny, "seed": seed})
    m.meta["u0"] = u0
    return m


# ---- configuration 4: two-phase RVE cubes ------------------------------------
def _sqdist(a, b):
    """Squared distances between the rows of a and of b, summed x, y, z in order."""
    dx = a[:, None, 0] - b[None, :, 0]
    dy = a[:, None, 1] - b[None, :, 1]
    dz = a[:, None, 2] - b[None, :, 2]
    return dx * dx + dy * dy + dz * dz


def _place_spheres(CC, R, vf_target, block=256):
    """Sequential random addition: candidate t is accepted when it overlaps no
    sphere accepted before it, until the accepted volume reaches vf_target.
    Candidates are screened in blocks against the spheres accepted before the
    block (vectorised); survivors are then checked in order against the ones
    accepted inside the block, which gives exactly the sequential result."""
    acc_c = np.zeros((0, 3))
    acc_r = np.zeros(0)
    vol = 0.0
    for b0 in range(0, len(R), block):
        if vol >= vf_target:
            break
        cb, rb = CC[b0:b0 + block], R[b0:b0 + block]
        if acc_r.size:
            d = np.sqrt(_sqdist(cb, acc_c))
            ok = ~np.any(d < rb[:, None] + acc_r[None, :], axis=1)
        else:
            ok = np.ones(len(rb), bool)
        cand = np.flatnonzero(ok)
        cc, rr = cb[cand], rb[cand]
        ov = (np.sqrt(_sqdist(cc, cc)) < rr[:, None] + rr[None, :]).tolist()
        taken = []
        for a in range(len(cand)):
            if vol >= vf_target:
                break
            row = ov[a]
            if any(row[q] for q in taken):
                continue
            taken.append(a)
            vol += 4.0 / 3.0 * math.pi * float(rr[a]) ** 3
        if taken:
            acc_c = np.vstack([acc_c, cc[taken]])
            acc_r = np.append(acc_r, rr[taken])
    return acc_c, acc_r


def _mark_inclusions(n, centres, radii):
    """Elements of the n^3 unit-cube grid whose centre lies inside a sphere
    (each sphere visits only the element block of its bounding box)."""
    h = 1.0 / n
    g = (np.arange(n) + 0.5) * h  # element-centre coordinates along each axis
    inc = np.zeros((n, n, n), bool)  # [k, j, i] = element i + n*(j + n*k)
    for c, r in zip(centres, radii):
        lo = np.maximum(np.floor((c - r) / h - 0.5).astype(int), 0)
        hi = np.minimum(np.ceil((c + r) / h - 0.5).astype(int) + 1, n)
        dx = (g[lo[0]:hi[0]] - c[0]) ** 2
        dy = (g[lo[1]:hi[1]] - c[1]) ** 2
        dz = (g[lo[2]:hi[2]] - c[2]) ** 2
        inside = dz[:, None, None] + dy[None, :, None] + dx[None, None, :] <= r * r
        inc[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]] |= inside
    return inc.ravel()


def rve_hex8(n, seed, order=2, E_matrix=1e3, contrast=10.0, nu=0.3, ux=0.01):
    """n^3 hex8 unit cube with non-overlapping spherical inclusions placed by
    seeded rejection until the drawn volume fraction ~U[0.2,0.4] is reached
    (radii ~U[0.05,0.15]); E_incl = contrast*E_matrix; x=0 clamped, u_x = ux on x=1."""
    xyz, conn = grid_hex8(n, n, n)
    vf_target = 0.2 + 0.2 * uniform(seed, 11, 0)[()]
    tries = np.arange(20000, dtype=np.uint64)
    R = 0.05 + 0.10 * uniform(seed, 12, tries)
    CC = np.stack([uniform(seed, 13, tries), uniform(seed, 14, tries), uniform(seed, 15, tries)], axis=1)
    CC = R[:, None] + (1 - 2 * R[:, None]) * CC
    centres, radii = _place_spheres(CC, R, vf_target)
    inc = _mark_inclusions(n, centres, radii)
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


# ---- configuration 5: serving request stream ----------------------------------
SERVE_FAMILIES = ("quad4_pstress", "hex8_elastic", "hex8_heat")


def serve_request(seed, i, dof_lo=1e3, dof_hi=5e5):
    """Request i of a seeded serving stream.  Element family uniform over quad4
    plane stress, hex8 elasticity and hex8 steady diffusion; size log-uniform
    in [dof_lo, dof_hi] dofs; box aspect ratios ~U[0.5, 2] with cubic cells of
    side h = 1/nx (seeded geometry); per-element lognormal moduli as the cube
    (E = 1e4 exp(N(0, 0.5^2)), nu ~ U[0.20, 0.35]) or conductivity
    k = exp(N(0, 1)).  Loads: quad4 -- left edge clamped, unit +x traction on
    the right edge; hex8 elasticity -- z=0 clamped, unit pressure on the top;
    diffusion -- T = 1 on x=0 and T = 0 on x=lx."""
    rs = seed * 1000003 + i
    fam = int(uniform(rs, 31, 0)[()] * 3) % 3
    target = math.exp(math.log(dof_lo) + (math.log(dof_hi) - math.log(dof_lo)) * uniform(rs, 32, 0)[()])
    a = 0.5 * 4.0 ** uniform(rs, 33, 0)[()]
    b = 0.5 * 4.0 ** uniform(rs, 34, 0)[()]
    if fam == 0:  # 2 (nx+1)(ny+1) ~ target
        nx = max(2, int(round(math.sqrt(target / 2.0 / a))) - 1)
        ny = max(2, int(round(nx * a)))
        xyz, conn = grid_quad4(nx, ny, 1.0, ny / nx)
        ne = conn.shape[0]
        eid = np.arange(ne, dtype=np.uint64)
        params = pstress_params(1e4 * np.exp(0.5 * normal(rs, 1, eid)), 0.20 + 0.15 * uniform(rs, 3, eid))
        ndof = 2 * xyz.shape[0]
        rest = np.zeros(ndof, np.uint8)
        left = np.where(np.isclose(xyz[:, 0], 0.0))[0]
        rest[2 * left] = 1
        rest[2 * left + 1] = 1
        right = np.where(np.isclose(xyz[:, 0], 1.0))[0]
        h = 1.0 / nx
        w = np.full(right.shape, h)
        w[np.isclose(xyz[right, 1], 0.0) | np.isclose(xyz[right, 1], ny / nx)] = h / 2
        load = np.zeros(ndof)
        load[2 * right] = w
        return Model(f"serve_{i}_quad4_{nx}x{ny}", _abi.QUAD4_PSTRESS, 2, xyz, conn, 2, params, rest,
                     np.zeros(ndof), load, 2, {"family": SERVE_FAMILIES[fam], "i": i, "seed": seed})
    ndpn = 3 if fam == 1 else 1
    nx = max(2, int(round((target / ndpn / (a * b)) ** (1.0 / 3.0))) - 1)
    ny, nz = max(2, int(round(nx * a))), max(2, int(round(nx * b)))
    lx, ly, lz = 1.0, ny / nx, nz / nx
    xyz, conn = grid_hex8(nx, ny, nz, lx, ly, lz)
    ne = conn.shape[0]
    eid = np.arange(ne, dtype=np.uint64)
    nnode = xyz.shape[0]
    if fam == 1:
        params = iso3d_params(1e4 * np.exp(0.5 * normal(rs, 1, eid)), 0.20 + 0.15 * uniform(rs, 3, eid))
        ndof = 3 * nnode
        rest = np.zeros(ndof, np.uint8)
        bot = np.where(np.isclose(xyz[:, 2], 0.0))[0]
        for c in range(3):
            rest[3 * bot + c] = 1
        top = np.where(np.isclose(xyz[:, 2], lz))[0]
        h = 1.0 / nx
        onx = np.isclose(xyz[top, 0], 0.0) | np.isclose(xyz[top, 0], lx)
        ony = np.isclose(xyz[top, 1], 0.0) | np.isclose(xyz[top, 1], ly)
        nface = 4 // (1 + onx.astype(int)) // (1 + ony.astype(int))
        load = np.zeros(ndof)
        load[3 * top + 2] = -h * h / 4.0 * nface
        return Model(f"serve_{i}_hex8_{nx}x{ny}x{nz}", _abi.HEX8_ELASTIC, 3, xyz, conn, 3, params, rest,
                     np.zeros(ndof), load, 2, {"family": SERVE_FAMILIES[fam], "i": i, "seed": seed})
    k = np.exp(normal(rs, 5, eid))
    params = np.stack([k, k, k, np.ones(ne)], axis=1)
    x0 = np.isclose(xyz[:, 0], 0.0)
    x1 = np.isclose(xyz[:, 0], lx)
    rest = (x0 | x1).astype(np.uint8)
    presc = np.where(x0, 1.0, 0.0)
    return Model(f"serve_{i}_heat_{nx}x{ny}x{nz}", _abi.HEX8_HEAT, 3, xyz, conn, 1, params, rest, presc,
                 np.zeros(nnode), 2, {"family": SERVE_FAMILIES[fam], "i": i, "seed": seed})
