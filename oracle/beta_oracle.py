"""ctypes view of the CPU oracle (test infrastructure only).

The oracle is a C++ FP64 restatement of BETA's assembly + Jacobi-PCG path
(``beta_oracle.cpp``).  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` import this module; the GPU product never
does.  ``RefLeaf`` wraps the reference's own ``gauss.cpp``/``shape.cpp``
compiled into ``_ref/`` (present only where the reference tree was available
at build time).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libbeta_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libbeta_ref_leaf.so")
REF_MATERIAL_LIB = os.path.join(HERE, "_ref", "libbeta_ref_material.so")
REF_EQUATIONS_LIB = os.path.join(HERE, "_ref", "libbeta_ref_equations.so")

KIND_QUAD4_PSTRESS = 1
KIND_HEX8_ELASTIC = 2
KIND_HEX8_HEAT = 3

OK = 0
ERR_MAXIT = 4
ERR_NEG_DIAG = 6
ERR_ZERO_DIAG = 7
ERR_LOAD_ON_RESTRAINED = 12


def build() -> None:
    """Compile the oracle (and _ref when the reference tree is present)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_lp = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_up = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


class SolveStats(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int), ("last_norm", C.c_double)]


def _load():
    if not os.path.exists(LIB):
        build()
    lib = C.CDLL(LIB)
    V, I, D, P = C.c_void_p, C.c_int, C.c_double, C.c_void_p
    sig = {
        "oracle_gauss_1d": (I, [I, _dp, _dp]),
        "oracle_hex_points": (I, [I, _dp, _dp, _dp, _dp]),
        "oracle_quad_points": (I, [I, _dp, _dp, _dp]),
        "oracle_shape_hex8": (None, [D, D, D, _dp, _dp, _dp, _dp]),
        "oracle_shape_quad4": (None, [D, D, _dp, _dp, _dp]),
        "oracle_invert": (I, [I, _dp]),
        "oracle_cmat_ortho3d": (I, [_dp, _dp]),
        "oracle_cmat_plane_stress": (None, [_dp, _dp]),
        "oracle_ke_hex8": (I, [_dp, _dp, I, _dp]),
        "oracle_ke_quad4": (I, [_dp, _dp, I, _dp]),
        "oracle_km_hex8_heat": (I, [_dp, _dp, D, I, _dp, _dp]),
        "oracle_km_quad4_heat": (I, [_dp, _dp, D, I, _dp, _dp]),
        "oracle_fe_hex8": (I, [_dp, _dp, I, _dp, _dp]),
        "oracle_gnl_hex8": (I, [_dp, _dp, I, _dp, P, P]),
        "oracle_sys_assemble_gnl": (I, [V, I, _ip, _dp, _ip, _dp, I, _dp]),
        "oracle_fint_gnl": (I, [I, _ip, _dp, _ip, _dp, I, _dp, _dp, I]),
        "oracle_newton_hex8": (I, [V, I, _ip, _dp, _ip, _dp, I, _dp, D, I, D, I, _dp, C.POINTER(C.c_int),
                                   C.POINTER(C.c_int)]),
        "oracle_sys_create": (V, [I]),
        "oracle_sys_destroy": (None, [V]),
        "oracle_sys_set_zero_diag": (None, [V, D]),
        "oracle_sys_set_bc": (I, [V, _up, _dp, _dp]),
        "oracle_sys_specify": (None, [V, _ip, I]),
        "oracle_sys_allocate": (None, [V]),
        "oracle_sys_zero": (None, [V]),
        "oracle_sys_nnz": (C.c_longlong, [V]),
        "oracle_sys_add_matrix": (I, [V, _dp, _ip, I, P]),
        "oracle_sys_export_lower": (None, [V, _lp, _ip, _dp]),
        "oracle_sys_pseudo_load": (None, [V, _dp]),
        "oracle_sys_vector_product": (None, [V, _dp, _dp]),
        "oracle_sys_solve": (I, [V, P, D, I, _dp, C.POINTER(SolveStats)]),
        "oracle_sys_rhs": (None, [V, _dp]),
        "oracle_sys_specify_mesh": (None, [V, I, I, I, _ip, _ip]),
        "oracle_sys_assemble_mesh": (I, [V, I, I, I, I, I, _ip, _dp, _ip, _dp, I, I]),
        "oracle_sys_assemble_mesh_threaded": (I, [V, I, I, I, I, I, _ip, _dp, _ip, _dp, I, I, I]),
        "oracle_internal_force_hex8": (I, [I, _ip, _dp, _ip, _dp, I, P, _dp, _dp]),
        "oracle_element_outputs": (I, [I, I, _ip, _dp, _ip, _dp, I, _dp, _dp]),
        "oracle_heat_step": (I, [V, I, I, _ip, _dp, _ip, _dp, I, D, D, _dp, D, I, C.POINTER(SolveStats)]),
        "oracle_csr_from_sys": (V, [V]),
        "oracle_csr_destroy": (None, [V]),
        "oracle_csr_pcg_threaded": (I, [V, _dp, _dp, D, I, I, C.POINTER(SolveStats)]),
        "oracle_csr_pcg_threaded_rule": (I, [V, _dp, _dp, D, I, I, I, P, I, C.POINTER(SolveStats)]),
        "oracle_csr_from_lower": (V, [I, _lp, _ip, _dp]),
        "oracle_cmat_ortho3d_many": (I, [I, _dp, _dp]),
        "oracle_element_matrices_threaded": (I, [I, I, I, I, I, _ip, _dp, _dp, I, I, I, _dp, I]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        _LIB = _load()
    return _LIB


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


# -- element level ---------------------------------------------------------
def gauss_1d(k):
    x, w = np.zeros(k), np.zeros(k)
    assert lib().oracle_gauss_1d(k, x, w) == 0
    return x, w


def hex_points(order):
    n = order ** 3
    a = [np.zeros(n) for _ in range(4)]
    assert lib().oracle_hex_points(order, *a) == 0
    return a


def quad_points(order):
    n = order ** 2
    a = [np.zeros(n) for _ in range(3)]
    assert lib().oracle_quad_points(order, *a) == 0
    return a


def shape_hex8(xi, eta, zeta):
    S, d0, d1, d2 = (np.zeros(8) for _ in range(4))
    lib().oracle_shape_hex8(xi, eta, zeta, S, d0, d1, d2)
    return S, d0, d1, d2


def shape_quad4(xi, eta):
    S, d0, d1 = (np.zeros(4) for _ in range(3))
    lib().oracle_shape_quad4(xi, eta, S, d0, d1)
    return S, d0, d1


def invert(A):
    A = _f64(A).copy()
    n = A.shape[0]
    st = lib().oracle_invert(n, A.reshape(-1))
    if st:
        raise ArithmeticError(f"singular matrix (status {st})")
    return A


def cmat_ortho3d(m9):
    C36 = np.zeros(36)
    assert lib().oracle_cmat_ortho3d(_f64(m9), C36) == 0
    return C36.reshape(6, 6)


def cmat_ortho3d_many(params):
    """cmat_ortho3d for every row of params (n x 9): n x 6 x 6."""
    params = _f64(params)
    out = np.zeros((params.shape[0], 36))
    assert lib().oracle_cmat_ortho3d_many(params.shape[0], params.reshape(-1), out.reshape(-1)) == 0
    return out.reshape(-1, 6, 6)


def cmat_plane_stress(m4):
    C9 = np.zeros(9)
    lib().oracle_cmat_plane_stress(_f64(m4), C9)
    return C9.reshape(3, 3)


def _full_from_upper(Ku):
    return np.triu(Ku) + np.triu(Ku, 1).T


def ke_hex8(xyz, C36, order=2):
    Ke = np.zeros(24 * 24)
    st = lib().oracle_ke_hex8(_f64(xyz).reshape(-1), _f64(C36).reshape(-1), order, Ke)
    return st, _full_from_upper(Ke.reshape(24, 24))


def ke_quad4(xy, C9, order=2):
    Ke = np.zeros(64)
    st = lib().oracle_ke_quad4(_f64(xy).reshape(-1), _f64(C9).reshape(-1), order, Ke)
    return st, _full_from_upper(Ke.reshape(8, 8))


def km_hex8_heat(xyz, k3, c, order=2):
    """hex8 diffusion K and M (full 8x8); k3: (k11, k22, k33) or a full 3x3
    conductivity."""
    K, M = np.zeros(64), np.zeros(64)
    k = np.asarray(k3, dtype=np.float64)
    k9 = (np.diag(k) if k.ndim == 1 else k).reshape(-1).copy()
    st = lib().oracle_km_hex8_heat(_f64(xyz).reshape(-1), _f64(k9), float(c), order, K, M)
    return st, _full_from_upper(K.reshape(8, 8)), _full_from_upper(M.reshape(8, 8))


def km_quad4_heat(xy, k2, c, order=2):
    """quad4 diffusion K and M (full 4x4) for conductivities k2 = (k11, k22)."""
    K, M = np.zeros(16), np.zeros(16)
    k4 = np.diag(np.asarray(k2, dtype=np.float64)).reshape(-1)
    st = lib().oracle_km_quad4_heat(_f64(xy).reshape(-1), _f64(k4), float(c), order, K, M)
    return st, _full_from_upper(K.reshape(4, 4)), _full_from_upper(M.reshape(4, 4))


def fe_hex8(xyz, C36, ue, order=2):
    Fe = np.zeros(24)
    assert lib().oracle_fe_hex8(_f64(xyz).reshape(-1), _f64(C36).reshape(-1), order, _f64(ue), Fe) == 0
    return Fe


# -- system level ----------------------------------------------------------
class System:
    """Equations + SymmetricSparseMatrix restated (default 'SPARSE' storage)."""

    def __init__(self, mesh):
        self.mesh = mesh
        self.n = int(mesh.ndof)
        self.h = lib().oracle_sys_create(self.n)
        if not self.h:
            raise ValueError("empty system")
        self._csr = None

    def __del__(self):
        try:
            if self._csr:
                lib().oracle_csr_destroy(self._csr)
            if self.h:
                lib().oracle_sys_destroy(self.h)
        except Exception:
            pass

    def set_bc(self, restrained, prescribed, load):
        st = lib().oracle_sys_set_bc(self.h, np.ascontiguousarray(restrained, dtype=np.uint8),
                                     _f64(prescribed), _f64(load))
        return st

    def build_pattern(self):
        m = self.mesh
        lib().oracle_sys_specify_mesh(self.h, m.nelem, m.nnpe, m.ndpn, _i32(m.conn).reshape(-1),
                                      _i32(m.first_dof))
        lib().oracle_sys_allocate(self.h)
        return int(lib().oracle_sys_nnz(self.h))

    def assemble(self, params, order):
        m = self.mesh
        params = _f64(params)
        return lib().oracle_sys_assemble_mesh(
            self.h, m.kind, m.nelem, m.nnpe, m.ndpn, m.ndim, _i32(m.conn).reshape(-1),
            _f64(m.xyz).reshape(-1), _i32(m.first_dof), params.reshape(-1), params.shape[1], order)

    def assemble_threaded(self, params, order, threads=0):
        """assemble() with the element matrices computed on all threads and
        added in element order: the same system, bit for bit."""
        m = self.mesh
        params = _f64(params)
        return lib().oracle_sys_assemble_mesh_threaded(
            self.h, m.kind, m.nelem, m.nnpe, m.ndpn, m.ndim, _i32(m.conn).reshape(-1),
            _f64(m.xyz).reshape(-1), _i32(m.first_dof), params.reshape(-1), params.shape[1], order, int(threads))

    def csr(self):
        """The threaded solver's full CSR of this system."""
        rp, col, val = self.export_lower()
        return Csr(self.n, rp, col, val)

    def export_lower(self):
        nnz = int(lib().oracle_sys_nnz(self.h))
        rp = np.zeros(self.n + 1, dtype=np.int64)
        col = np.zeros(nnz, dtype=np.int32)
        val = np.zeros(nnz)
        lib().oracle_sys_export_lower(self.h, rp, col, val)
        return rp, col, val

    def pseudo_load(self):
        out = np.zeros(self.n)
        lib().oracle_sys_pseudo_load(self.h, out)
        return out

    def rhs(self):
        out = np.zeros(self.n)
        lib().oracle_sys_rhs(self.h, out)
        return out

    def matvec(self, x):
        y = np.zeros(self.n)
        lib().oracle_sys_vector_product(self.h, _f64(x), y)
        return y

    def set_zero_diag(self, value):
        """Replacement for zero diagonals at the solve (0: a zero diagonal is
        an error, as in the reference without ReplaceZeroDiagonal)."""
        lib().oracle_sys_set_zero_diag(self.h, float(value))

    def solve(self, eps=1e-4, maxit=10000, init_guess=None):
        out = np.zeros(self.n)
        st = SolveStats()
        g = None if init_guess is None else _f64(init_guess)
        rc = lib().oracle_sys_solve(self.h, None if g is None else g.ctypes.data, eps, maxit, out,
                                    C.byref(st))
        return rc, out, st

    def solve_threaded(self, b, eps, maxit=10000, threads=0, x0=None):
        if self._csr is None:
            self._csr = lib().oracle_csr_from_sys(self.h)
        x = np.zeros(self.n) if x0 is None else _f64(x0).copy()
        st = SolveStats()
        rc = lib().oracle_csr_pcg_threaded(self._csr, _f64(b), x, eps, maxit, threads, C.byref(st))
        return rc, x, st

    def assemble_gnl(self, params, order, u):
        """The geometric-nonlinear tangent at total displacement u (hex8)."""
        m = self.mesh
        return lib().oracle_sys_assemble_gnl(self.h, m.nelem, _i32(m.conn).reshape(-1), _f64(m.xyz).reshape(-1),
                                             _i32(m.first_dof), _f64(params).reshape(-1), int(order), _f64(u))

    def newton(self, params, order, u0, max_residual=1e-10, max_newton=400, eps=1e-10, maxit=100000):
        """BasicModel::iterate for hex8 elasticity (geometric nonlinear) from
        the total displacement u0: (rc, u, history of max |R| per iteration,
        Newton solves, PCG iterations in all)."""
        m = self.mesh
        u = _f64(u0).copy()
        hist = np.zeros(max_newton + 1)
        its, lin = C.c_int(0), C.c_int(0)
        rc = lib().oracle_newton_hex8(self.h, m.nelem, _i32(m.conn).reshape(-1), _f64(m.xyz).reshape(-1),
                                      _i32(m.first_dof), _f64(params).reshape(-1), int(order), u,
                                      float(max_residual), int(max_newton), float(eps), int(maxit), hist,
                                      C.byref(its), C.byref(lin))
        return rc, u, hist[:its.value + 1], its.value, lin.value

    def heat_step(self, params, order, dt, u_s, alpha=1.0, eps=1e-10, maxit=10000):
        m = self.mesh
        st = SolveStats()
        u = _f64(u_s).copy()
        rc = lib().oracle_heat_step(self.h, m.kind, m.nelem, _i32(m.conn).reshape(-1), _f64(m.xyz).reshape(-1),
                                    _i32(m.first_dof), _f64(params).reshape(-1), order, dt, alpha, u,
                                    eps, maxit, C.byref(st))
        return rc, u, st


def gnl_hex8(xyz, C36, ue, order=2):
    """Geometric-nonlinear hex8 at nodal displacements ue (24): (tangent Ke
    24 x 24 upper triangle, Fe 24) -- ElasticityElement3D with analysisType
    GEOMETRIC_NONLINEAR."""
    Ke, Fe = np.zeros(576), np.zeros(24)
    st = lib().oracle_gnl_hex8(_f64(xyz).reshape(-1), _f64(C36).reshape(-1), int(order), _f64(ue).reshape(-1),
                               Ke.ctypes.data, Fe.ctypes.data)
    if st:
        raise ArithmeticError(f"gnl_hex8 status {st}")
    return Ke.reshape(24, 24), Fe


def internal_force_gnl_hex8(mesh, params, order, u):
    """sum_e Fe(u) of the geometric-nonlinear hex8 element over all rows."""
    f = np.zeros(mesh.ndof)
    st = lib().oracle_fint_gnl(mesh.nelem, _i32(mesh.conn).reshape(-1), _f64(mesh.xyz).reshape(-1),
                               _i32(mesh.first_dof), _f64(params).reshape(-1), int(order), _f64(u), f, mesh.ndof)
    assert st == 0
    return f


def internal_force_hex8(mesh, params, order, u, restrained=None):
    f = np.zeros(mesh.ndof)
    r = None if restrained is None else np.ascontiguousarray(restrained, dtype=np.uint8)
    st = lib().oracle_internal_force_hex8(mesh.nelem, _i32(mesh.conn).reshape(-1), _f64(mesh.xyz).reshape(-1),
                                          _i32(mesh.first_dof), _f64(params).reshape(-1), order,
                                          None if r is None else r.ctypes.data, _f64(u), f)
    assert st == 0
    return f


def element_outputs(mesh, params, order, u):
    """Per element [volume, int stress dV, int strain dV, strain energy]
    (ElasticityElement3D::getVolAvgValues), hex8 (6 components) or quad4 (3)."""
    ns = 6 if mesh.kind == 2 else 3
    out = np.zeros((mesh.nelem, 2 * ns + 2))
    st = lib().oracle_element_outputs(mesh.kind, mesh.nelem, _i32(mesh.conn).reshape(-1), _f64(mesh.xyz).reshape(-1),
                                      _i32(mesh.first_dof), _f64(params).reshape(-1), order, _f64(u), out)
    assert st == 0
    return out


def element_matrices_threaded(mesh, params, order, e0, e1, threads=0):
    nd = mesh.nnpe * mesh.ndpn
    out = np.zeros((e1 - e0) * nd * nd)
    params = _f64(params)
    st = lib().oracle_element_matrices_threaded(mesh.kind, e0, e1, mesh.nnpe, mesh.ndim,
                                                _i32(mesh.conn).reshape(-1), _f64(mesh.xyz).reshape(-1),
                                                params.reshape(-1), params.shape[1], order, nd, out, threads)
    return st, out


class Csr:
    """The threaded Jacobi-PCG's full CSR built from a lower triangle (0-based
    CSR rows, as SymmetricSparseMatrix stores it)."""

    RULE_REF, RULE_RB = 0, 1

    def __init__(self, n, rp, col, val):
        self.n = int(n)
        self.h = lib().oracle_csr_from_lower(self.n, np.ascontiguousarray(rp, np.int64), _i32(col), _f64(val))

    def __del__(self):
        try:
            if self.h:
                lib().oracle_csr_destroy(self.h)
        except Exception:
            pass

    def pcg(self, b, eps, maxit=100000, threads=0, rule=0, x0=None, trace_len=0):
        """Jacobi-PCG from x0 (zero) to sqrt(r.r/x.x) < eps (rule 0, the
        reference's) or sqrt(r.r/b.b) < eps (rule 1).  Returns (rc, x, stats,
        trace): trace holds the reference rule's quantity after each of the
        first trace_len iterations."""
        x = np.zeros(self.n) if x0 is None else _f64(x0).copy()
        st = SolveStats()
        tr = np.zeros(max(1, trace_len))
        rc = lib().oracle_csr_pcg_threaded_rule(self.h, _f64(b), x, float(eps), int(maxit), int(threads), int(rule),
                                                tr.ctypes.data if trace_len else None, int(trace_len), C.byref(st))
        return rc, x, st, tr[:min(trace_len, st.iterations)]


# -- setElementMaterial block of an input deck ----------------------------------
def element_groups_from_block(text, nelem, init=-1):
    """BasicModel::ProcessSetElementProperty (BasicModel.cpp:682-775) for the
    material command, lines read as getLineAndTokenize does
    (getLineAndTokenize.cpp:210-237: blank/tab tokens, comments stripped,
    empty lines skipped, case-insensitive terminator "end").  Returns the
    group per element, or None where the reference's input would be
    refused or undefined."""
    import re
    body = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    if "/*" in body:
        return None
    g = [init] * nelem
    for line in body.split("\n"):
        tok = line.split("//")[0].replace("\r", " ").split()
        if not tok:
            continue
        if tok[0].lower() == "end":
            break
        try:
            if len(tok) >= 2 and tok[0].lower() == "all":
                first, last, inc, grp = 0, nelem - 1, 1, int(tok[1])
            else:
                first = int(tok[0])
                if first < 0:
                    break
                if len(tok) < 4:
                    return None
                last, inc, grp = int(tok[1]), int(tok[2]), int(tok[3])
        except ValueError:
            return None
        if first > last or last >= nelem or inc < 1 or grp < 0:
            return None
        for e in range(first, last + 1, inc):
            g[e] = grp
    return g


# -- SurfaceLoad::applyTo flux integration ------------------------------------
# Restated from beta/BCs/SurfaceLoad.cpp:16-255 (without the shared-memory
# coupling that supplies the nodal fluxes there): per surface element, the
# nodal flux is interpolated to each integration point, the surface scale
# |g| = |dx/dxi x dx/deta| is formed, and w * q(xi) * N_i * |g| is added to
# the first dof of node i.  4- and 8-node quadrilaterals use the 3x3 Gauss
# rule (SurfaceLoad.cpp:66-99), 6-node triangles the 7-point rule with the
# weights halved (SurfaceLoad.cpp:100-139).  Shapes: beta/elements/shape.cpp
# (shapeQuad4 / shapeQuad8 / shapeTri6 and their derivatives, node orders
# as there).
_G3 = 0.774596669241483
SURF_QUAD_RULE = (np.array([_G3, 0.0, -_G3] * 3), np.repeat([_G3, 0.0, -_G3], 3),
                  np.array([25, 40, 25, 40, 64, 40, 25, 40, 25], dtype=float) / 81.0)
_T7 = (0.101286507323, 0.797426985353, 0.470142064105, 0.059715871789)
SURF_TRI_RULE = (np.array([1.0 / 3, _T7[0], _T7[0], _T7[1], _T7[2], _T7[2], _T7[3]]),
                 np.array([1.0 / 3, _T7[0], _T7[1], _T7[0], _T7[2], _T7[3], _T7[2]]),
                 0.5 * np.array([0.225] + [0.125939180544] * 3 + [0.132394152788] * 3))


def surface_shape(npe, xi, eta):
    """(N, dN/dxi, dN/deta) of a 4-node quad, 8-node quad or 6-node triangle."""
    if npe == 4:
        sx, se = np.array([-1.0, 1.0, 1.0, -1.0]), np.array([-1.0, -1.0, 1.0, 1.0])
        N = 0.25 * (1 + sx * xi) * (1 + se * eta)
        return N, 0.25 * sx * (1 + se * eta), 0.25 * se * (1 + sx * xi)
    if npe == 8:
        # corner, mid-side, corner, ... counter-clockwise from (-1, -1)
        px = np.array([-1.0, 0.0, 1.0, 1.0, 1.0, 0.0, -1.0, -1.0])
        pe = np.array([-1.0, -1.0, -1.0, 0.0, 1.0, 1.0, 1.0, 0.0])
        N, dx, de = np.zeros(8), np.zeros(8), np.zeros(8)
        for i in range(8):
            a, b = px[i], pe[i]
            if a != 0 and b != 0:  # corner
                N[i] = 0.25 * (1 + a * xi) * (1 + b * eta) * (a * xi + b * eta - 1)
                dx[i] = 0.25 * a * (1 + b * eta) * (2 * a * xi + b * eta)
                de[i] = 0.25 * b * (1 + a * xi) * (a * xi + 2 * b * eta)
            elif a == 0:  # mid-side on eta = b
                N[i] = 0.5 * (1 - xi * xi) * (1 + b * eta)
                dx[i] = -xi * (1 + b * eta)
                de[i] = 0.5 * b * (1 - xi * xi)
            else:  # mid-side on xi = a
                N[i] = 0.5 * (1 + a * xi) * (1 - eta * eta)
                dx[i] = 0.5 * a * (1 - eta * eta)
                de[i] = -eta * (1 + a * xi)
        return N, dx, de
    if npe == 6:
        l0 = 1 - xi - eta  # area coordinates (l0, xi, eta); corner, mid-side, ...
        N = np.array([l0 * (2 * l0 - 1), 4 * xi * l0, xi * (2 * xi - 1), 4 * xi * eta, eta * (2 * eta - 1),
                      4 * eta * l0])
        dx = np.array([1 - 4 * l0, 4 * (l0 - xi), 4 * xi - 1, 4 * eta, 0.0, -4 * eta])
        de = np.array([1 - 4 * l0, -4 * xi, 0.0, 4 * xi, 4 * eta - 1, 4 * (l0 - eta)])
        return N, dx, de
    raise ValueError("surface elements have 4, 6 or 8 nodes")


def surface_flux_load(surf_conn, xyz, nodal_flux, first_dof, ndof):
    """Nodal loads of a nodal surface flux (SurfaceLoad::applyTo)."""
    surf_conn = np.asarray(surf_conn)
    npe = surf_conn.shape[1]
    xs, es, ws = SURF_TRI_RULE if npe == 6 else SURF_QUAD_RULE
    F = np.zeros(ndof)
    for nodes in surf_conn:
        X = np.asarray(xyz, dtype=float)[nodes]
        q = np.asarray(nodal_flux, dtype=float)[nodes]
        fe = np.zeros(npe)
        for xi, eta, w in zip(xs, es, ws):
            N, dx, de = surface_shape(npe, xi, eta)
            gx, ge = dx @ X, de @ X
            modg = np.linalg.norm(np.cross(gx, ge))
            fe += w * (N @ q) * N * modg
        for i, nd in enumerate(nodes):
            F[first_dof[nd]] += fe[i]
    return F


# -- the reference's own leaf code (oracle/_ref) -----------------------------
class RefMaterial:
    """The reference's matrix.cpp, elastic.cpp and pStress.cpp, compiled
    unmodified: the constitutive matrices as the materials' own read()
    builds them from input constants, and the dense LU inverse."""

    def __init__(self):
        if not os.path.exists(REF_MATERIAL_LIB):
            raise FileNotFoundError(REF_MATERIAL_LIB)
        self.lib = C.CDLL(REF_MATERIAL_LIB)
        self.lib.ref_matrix_invert.argtypes = [C.c_int, _dp]
        self.lib.ref_cmat_ortho3d.argtypes = [_dp, _dp, C.c_void_p]
        self.lib.ref_cmat_plane_stress.argtypes = [_dp, _dp]
        self.lib.ref_elastic_stress.argtypes = [_dp, _dp, _dp]
        self.lib.ref_heat_conductivity.argtypes = [_dp, _dp, _dp, _dp]
        _ip32 = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
        self.lib.ref_set_num_dof.argtypes = [C.c_int, C.c_char_p, _ip32, _ip32, C.POINTER(C.c_int)]
        self.lib.ref_node_records.argtypes = [C.c_int, _ip32, _dp, C.c_char_p, _ip32, _dp]

    @staticmethod
    def available():
        return os.path.exists(REF_MATERIAL_LIB)

    def invert(self, A):
        """Matrix::invert of a square matrix."""
        A = np.ascontiguousarray(A, dtype=float)
        B = A.reshape(-1).copy()
        self.lib.ref_matrix_invert(A.shape[0], B)
        return B.reshape(A.shape)

    def cmat_ortho3d(self, m9):
        """ElasticMaterial read of readModuli (E11, E22, E33, nu12, nu23,
        nu13, G12, G23, G13): the 6 x 6 stiffness."""
        Cm = np.zeros(36)
        if self.lib.ref_cmat_ortho3d(_f64(m9), Cm, None):
            raise ValueError("ElasticMaterial::read failed")
        return Cm.reshape(6, 6)

    def cmat_plane_stress(self, m4):
        """PlaneStress read of (E11, E22, nu12, G12): the 3 x 3 stiffness."""
        Cm = np.zeros(9)
        if self.lib.ref_cmat_plane_stress(_f64(np.asarray(m4, dtype=float)[:4]), Cm):
            raise ValueError("PlaneStress::read failed")
        return Cm.reshape(3, 3)

    def set_num_dof(self, nnode, deck):
        """Node::setNumDofPerNode on nnode nodes reading deck: (numDof,
        firstDof, total)."""
        nd, fd, tot = np.zeros(nnode, np.int32), np.zeros(nnode, np.int32), C.c_int(0)
        self.lib.ref_set_num_dof(int(nnode), deck.encode(), nd, fd, C.byref(tot))
        return nd, fd, tot.value

    def node_records(self, nums, xyz, path):
        """Node::writeBinary of each node to path, then Node::readBinary of
        them back: (numbers, coordinates) as read."""
        nums = np.ascontiguousarray(nums, np.int32)
        xyz = _f64(xyz).reshape(-1, 3).copy()
        nb, xb = np.zeros_like(nums), np.zeros_like(xyz)
        if self.lib.ref_node_records(len(nums), nums, xyz.reshape(-1), str(path).encode(), nb, xb.reshape(-1)):
            raise OSError("ref_node_records could not write " + str(path))
        return nb, xb

    def heat_conductivity(self, k3, grad):
        """HeatTransferMaterial read of readConductivity (k11, k22, k33) and
        calculateFlux at the temperature gradient grad: (k 3 x 3, flux)."""
        Cm, flux = np.zeros(9), np.zeros(3)
        if self.lib.ref_heat_conductivity(_f64(k3), _f64(grad), Cm, flux):
            raise ValueError("HeatTransferMaterial::read failed")
        return Cm.reshape(3, 3), flux

    def elastic_stress(self, m9, strain):
        """ElasticMaterial::calculateStress at zero temperature and moisture."""
        out = np.zeros(6)
        if self.lib.ref_elastic_stress(_f64(m9), _f64(strain), out):
            raise ValueError("ElasticMaterial::read failed")
        return out


class RefEquations:
    """The reference's Equations (equation.cpp, addeqn.cpp) over its
    SymmetricSparseMatrix (sparse.cpp) and Matrix (matrix.cpp), compiled
    unmodified: the global pattern, addMatrix scatter with restraint
    elimination, loads and CG solve for given element matrices and maps."""

    def __init__(self):
        if not os.path.exists(REF_EQUATIONS_LIB):
            raise FileNotFoundError(REF_EQUATIONS_LIB)
        self.lib = C.CDLL(REF_EQUATIONS_LIB)
        _lp = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
        _ipc = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
        _u8 = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
        I, D = C.c_int, C.c_double
        self.lib.ref_equations_assemble.argtypes = [I, I, I, I, _ipc, _dp, C.c_void_p, _u8, _dp, _dp, D, I, C.c_void_p,
                                                    _lp, _ipc, _dp, C.c_longlong, C.POINTER(C.c_longlong), _dp, _dp,
                                                    C.c_void_p, _dp, D]
        self.lib.ref_equations_resultant.argtypes = [I, I, I, _ipc, _dp, _u8, _dp]

    @staticmethod
    def available():
        return os.path.exists(REF_EQUATIONS_LIB)

    def resultant(self, n, maps, Fe, restrained):
        """Equations::assembleResultantVector of element force vectors Fe
        (nelem x nde) with the restraint mask: the global internal force."""
        maps = np.ascontiguousarray(maps, dtype=np.int32)
        out = np.zeros(n)
        self.lib.ref_equations_resultant(n, maps.shape[0], maps.shape[1], maps.reshape(-1),
                                         _f64(Fe).reshape(-1).copy(), np.ascontiguousarray(restrained, np.uint8), out)
        return out

    def assemble(self, n, maps, Ke, restrained, prescribed, load, solve=False, eps=1e-4, maxit=10000, Fe=None,
                 x0=None, timings=None, parcg=False, zero_diag=0.0):
        """Element matrices Ke (and force vectors Fe) through the reference's
        Equations; solve from the initial guess x0 when asked.  Returns
        (rowptr, col, val, pseudo_load, load_vector, x or None); a list given
        as timings receives the seconds of structure, scatter and solve.
        parcg selects the reference's two-thread ParCG storage and solver
        instead of the default serial SymmetricSparseMatrix; zero_diag is the
        ReplaceZeroDiagonal option (0: none -- the reference then exits on a
        zero diagonal, so give one whenever a row can be empty)."""
        maps = np.ascontiguousarray(maps, dtype=np.int32)
        nelem, nde = maps.shape
        Ke = np.ascontiguousarray(Ke, dtype=float).reshape(-1)
        cap = nelem * nde * nde + n
        rp, col, val = np.zeros(n + 1, np.int64), np.zeros(cap, np.int32), np.zeros(cap)
        pseudo, lv = np.zeros(n), np.zeros(n)
        x = np.zeros(n) if solve else None
        nnz = C.c_longlong(0)
        fe = None if Fe is None else _f64(Fe).reshape(-1).copy()
        secs = np.zeros(3)
        g = None if x0 is None else _f64(x0).copy()
        rc = self.lib.ref_equations_assemble(int(bool(parcg)), n, nelem, nde, maps.reshape(-1), Ke,
                                             None if fe is None else fe.ctypes.data,
                                             np.ascontiguousarray(restrained, dtype=np.uint8), _f64(prescribed),
                                             _f64(load), float(eps), int(maxit), None if g is None else g.ctypes.data,
                                             rp, col, val, cap, C.byref(nnz), pseudo, lv,
                                             None if x is None else x.ctypes.data, secs, float(zero_diag))
        if rc:
            raise ValueError("ref_equations_assemble returned %d" % rc)
        k = nnz.value
        if timings is not None:
            timings[:] = secs.tolist()
        return rp, col[:k].copy(), val[:k].copy(), pseudo, lv, x


class RefSystem:
    """One full system held in the reference's own Equations (equation.cpp over
    SymmetricSparseMatrix, or ParCGMatrix when parcg), built in the
    reference's order by the calls below and solved repeatedly by
    Equations::solve: what the bench's reference arm times."""

    def __init__(self, n, restrained, prescribed, parcg=False, maxit=1000000):
        if not os.path.exists(REF_EQUATIONS_LIB):
            raise FileNotFoundError(REF_EQUATIONS_LIB)
        self.lib = C.CDLL(REF_EQUATIONS_LIB)
        L, V, I, D = self.lib, C.c_void_p, C.c_int, C.c_double
        _ipc = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
        _u8 = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
        for name, res, args in (
                ("ref_eqsys_create", V, [I, I, _u8, _dp, I]),
                ("ref_eqsys_pattern", I, [V, I, I, _ipc]),
                ("ref_eqsys_allocate", I, [V]),
                ("ref_eqsys_add", I, [V, I, I, _ipc, _dp]),
                ("ref_eqsys_loads", I, [V, _dp]),
                ("ref_eqsys_nnz", C.c_longlong, [V]),
                ("ref_eqsys_export", I, [V, _lp, _ipc, _dp, _dp]),
                ("ref_eqsys_solve", I, [V, D, V, V, C.POINTER(C.c_double)]),
                ("ref_eqsys_destroy", None, [V])):
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        self.n = int(n)
        self.h = L.ref_eqsys_create(int(bool(parcg)), self.n, np.ascontiguousarray(restrained, np.uint8),
                                    _f64(prescribed), int(maxit))

    def close(self):
        if self.h:
            self.lib.ref_eqsys_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def pattern(self, maps):
        maps = np.ascontiguousarray(maps, np.int32)
        self.lib.ref_eqsys_pattern(self.h, maps.shape[0], maps.shape[1], maps.reshape(-1))

    def allocate(self):
        self.lib.ref_eqsys_allocate(self.h)

    def add(self, maps, Ke):
        maps = np.ascontiguousarray(maps, np.int32)
        self.lib.ref_eqsys_add(self.h, maps.shape[0], maps.shape[1], maps.reshape(-1), _f64(Ke).reshape(-1))

    def loads(self, load):
        if self.lib.ref_eqsys_loads(self.h, _f64(load)):
            raise ValueError("a load sits on a restrained unknown")

    def nnz(self):
        return int(self.lib.ref_eqsys_nnz(self.h))

    def export(self):
        """(rp, col, val) of the lower triangle and the right-hand side b."""
        k = self.nnz()
        rp, col, val, b = np.zeros(self.n + 1, np.int64), np.zeros(k, np.int32), np.zeros(k), np.zeros(self.n)
        self.lib.ref_eqsys_export(self.h, rp, col, val, b)
        return rp, col, val, b

    def solve(self, eps, x0=None, want_x=False):
        """Equations::solve with stop tolerance eps from x0; returns (seconds,
        x or None).  The reference exits the process when its iteration
        limit is reached: choose eps so that it converges."""
        g = None if x0 is None else _f64(x0).copy()
        x = np.zeros(self.n) if want_x else None
        sec = C.c_double(0.0)
        self.lib.ref_eqsys_solve(self.h, float(eps), None if g is None else g.ctypes.data,
                                 None if x is None else x.ctypes.data, C.byref(sec))
        return sec.value, x


class RefLeaf:
    """The reference's gauss.cpp + shape.cpp, compiled unmodified."""

    def __init__(self):
        if not os.path.exists(REF_LIB):
            raise FileNotFoundError(REF_LIB)
        self.lib = C.CDLL(REF_LIB)
        I, D = C.c_int, C.c_double
        self.lib.ref_gauss_1d.argtypes = [I, _dp, _dp]
        self.lib.ref_hex_points.argtypes = [I, _dp, _dp, _dp, _dp]
        self.lib.ref_quad_points.argtypes = [I, _dp, _dp, _dp]
        self.lib.ref_shape_hex8.argtypes = [D, D, D, _dp, _dp, _dp, _dp]
        self.lib.ref_shape_quad4.argtypes = [D, D, _dp, _dp, _dp]
        self.lib.ref_shape_quad8.argtypes = [D, D, _dp, _dp, _dp]
        self.lib.ref_shape_tri6.argtypes = [D, D, _dp, _dp, _dp]
        self.lib.ref_sparse_solve_file.argtypes = [C.c_char_p, _dp, D, I, _dp, C.POINTER(C.c_int)]
        _lp = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
        _ipc = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
        self.lib.ref_print_lower.argtypes = [C.c_char_p, I, I, _lp, _ipc, _dp]
        self.lib.ref_heat2d_add_to_ke.argtypes = [D, D, D, I, _dp, _dp, D, _dp]
        self.lib.ref_heat3d_add_to_km.argtypes = [_dp, D, _dp, _dp, _dp, _dp, D, _dp, _dp]
        self.lib.ref_heat3d_step_terms.argtypes = [_dp, _dp, _dp, D, D, D, _dp, _dp]
        self.lib.ref_heat_step_terms.argtypes = [I, _dp, _dp, _dp, D, D, D, _dp, _dp]
        self.lib.ref_elastic_point.argtypes = [I, I, _dp, _dp, _dp, C.c_void_p, C.c_void_p, D, _dp, _dp, _dp]
        self.lib.ref_elastic_hex8_ke.argtypes = [I, _dp, _dp, I, _dp]
        self.lib.ref_heat_hex8_step_terms.argtypes = [I, _dp, _dp, _dp, I, _dp, D, D, D, _dp, _dp]
        self.lib.ref_elastic_quad4_ke.argtypes = [I, _dp, _dp, I, _dp]
        self.lib.ref_elastic_update.argtypes = [I, I, _dp, _dp, I, C.c_void_p, C.c_char_p, _dp, _dp, _dp]
        self.lib.ref_elastic_update_analysis.argtypes = [I, I, _dp, _dp, I, C.c_void_p, C.c_char_p, I, _dp, _dp,
                                                         _dp]
        self.lib.ref_elastic_vol_avg.argtypes = [I, I, _dp, _dp, I, _dp, _dp]
        self.lib.ref_heat_update.argtypes = [I, I, _dp, _dp, D, I, C.c_void_p, C.c_char_p, _dp, _dp]
        self.lib.ref_heat_hex8_k.argtypes = [I, _dp, _dp, I, _dp]
        self.lib.ref_write_csr.argtypes = [C.c_char_p, I, I, I, _ipc, _ipc, _dp]
        self.lib.ref_read_csr.argtypes = [C.c_char_p, I, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_void_p,
                                          C.c_void_p, C.c_void_p]

    @staticmethod
    def available():
        return os.path.exists(REF_LIB)

    def gauss_1d(self, k):
        x, w = np.zeros(k), np.zeros(k)
        self.lib.ref_gauss_1d(k, x, w)
        return x, w

    def hex_points(self, order):
        n = order ** 3
        a = [np.zeros(n) for _ in range(4)]
        self.lib.ref_hex_points(order, *a)
        return a

    def quad_points(self, order):
        n = order ** 2
        a = [np.zeros(n) for _ in range(3)]
        self.lib.ref_quad_points(order, *a)
        return a

    def shape_hex8(self, xi, eta, zeta):
        S, d0, d1, d2 = (np.zeros(8) for _ in range(4))
        self.lib.ref_shape_hex8(xi, eta, zeta, S, d0, d1, d2)
        return S, d0, d1, d2

    def shape_quad4(self, xi, eta):
        S, d0, d1 = (np.zeros(4) for _ in range(3))
        self.lib.ref_shape_quad4(xi, eta, S, d0, d1)
        return S, d0, d1

    def shape_quad8(self, xi, eta):
        S, d0, d1 = (np.zeros(8) for _ in range(3))
        self.lib.ref_shape_quad8(xi, eta, S, d0, d1)
        return S, d0, d1

    def shape_tri6(self, xi, eta):
        S, d0, d1 = (np.zeros(6) for _ in range(3))
        self.lib.ref_shape_tri6(xi, eta, S, d0, d1)
        return S, d0, d1

    def heat2d_add_to_ke(self, k11, k22, k12, dx, dy, factor, Ke):
        """HeatTransferElement2Dtransient::addToKe at one integration point;
        Ke (n x n, upper triangle) is accumulated in place."""
        n = len(dx)
        K = np.ascontiguousarray(Ke, dtype=np.float64).reshape(-1).copy()
        self.lib.ref_heat2d_add_to_ke(float(k11), float(k22), float(k12), n, np.ascontiguousarray(dx, dtype=float),
                                      np.ascontiguousarray(dy, dtype=float), float(factor), K)
        return K.reshape(n, n)

    def heat3d_add_to_km(self, k9, cap, S, dx, dy, dz, factor, K, M):
        """HeatTransferElement3Dtransient::addToKe + addToMe at one point;
        returns the accumulated (K, M) upper triangles (8 x 8)."""
        K = np.ascontiguousarray(K, dtype=float).reshape(-1).copy()
        M = np.ascontiguousarray(M, dtype=float).reshape(-1).copy()
        f = lambda a: np.ascontiguousarray(a, dtype=float)  # noqa: E731
        self.lib.ref_heat3d_add_to_km(f(np.asarray(k9).reshape(-1)), float(cap), f(S), f(dx), f(dy), f(dz),
                                      float(factor), K, M)
        return K.reshape(8, 8), M.reshape(8, 8)

    def heat_step_terms(self, K, M, u_s, a1, a2, dt):
        """formK_s and formF_s_new for an element of n = len(u_s) nodes (8:
        hex8, 4: quad4): (Mbar n x n, F n)."""
        n = len(u_s)
        Mb, F = np.zeros(n * n), np.zeros(n)
        f = lambda a: np.ascontiguousarray(a, dtype=float).reshape(-1)  # noqa: E731
        if self.lib.ref_heat_step_terms(n, f(K), f(M), f(u_s), float(a1), float(a2), float(dt), Mb, F):
            raise ValueError("ref_heat_step_terms: bad size")
        return Mb.reshape(n, n), F

    def heat3d_step_terms(self, K, M, u_s, a1, a2, dt):
        """formK_s and formF_s_new of the reference's 3D diffusion element:
        (Mbar 8 x 8, F 8)."""
        Mb, F = np.zeros(64), np.zeros(8)
        f = lambda a: np.ascontiguousarray(a, dtype=float).reshape(-1)  # noqa: E731
        self.lib.ref_heat3d_step_terms(f(K), f(M), f(u_s), float(a1), float(a2), float(dt), Mb, F)
        return Mb.reshape(8, 8), F

    def elastic_point(self, C_mat, dx, dy, dz, factor, Ke, u=None, Fe=None):
        """ElasticityElement3D (dz given) or ElasticityElement2D (dz None), the
        reference's own, at one integration point: calculateBmatrix + addToKe
        accumulated into Ke (upper triangle) and, for nodal displacements u
        (interleaved), derivativesOfFields + calculateStrain + addToFe of
        C * strain into Fe.  Returns (Ke, Fe, strain)."""
        dim = 2 if dz is None else 3
        n = len(dx)
        f = lambda a: np.ascontiguousarray(a, dtype=float).reshape(-1).copy()  # noqa: E731
        K = f(Ke)
        F = f(np.zeros(dim * n) if Fe is None else Fe)
        eps = np.zeros(6)
        dzv = None if dz is None else f(dz)
        uv = None if u is None else f(u)
        rc = self.lib.ref_elastic_point(dim, n, f(C_mat), f(dx), f(dy),
                                        None if dzv is None else dzv.ctypes.data,
                                        None if uv is None else uv.ctypes.data, float(factor), K, F, eps)
        if rc:
            raise ValueError("ref_elastic_point refused the element size")
        return K.reshape(dim * n, dim * n), F, eps[:3 if dim == 2 else 6]

    def elastic_hex8_ke(self, xyz, C36, order):
        """Hex8 stiffness (upper triangles, nel x 24 x 24) of elements xyz
        (nel x 8 x 3) with constitutive matrices C36 (nel x 6 x 6) through the
        reference's Gauss rule, shape functions and ElasticityElement3D B and
        addToKe (a serial loop)."""
        xyz = _f64(xyz).reshape(-1, 24)
        nel = xyz.shape[0]
        Ke = np.zeros(nel * 576)
        rc = self.lib.ref_elastic_hex8_ke(nel, xyz.reshape(-1).copy(), _f64(C36).reshape(-1).copy(), int(order), Ke)
        if rc:
            raise ValueError("ref_elastic_hex8_ke: non-positive Jacobian")
        return Ke.reshape(nel, 24, 24)

    def elastic_update_gnl(self, X, C_mat, order, action, u):
        """elastic_update with analysisType GEOMETRIC_NONLINEAR (the element of
        BasicModel::iterate): (Ke upper triangle, Fe, integrals)."""
        X = _f64(X)
        dim, nnode = X.shape[1], X.shape[0]
        n = dim * nnode
        Ke, Fe, sums = np.zeros(n * n), np.zeros(n), np.zeros(18)
        uv = _f64(u).reshape(-1).copy()
        rc = self.lib.ref_elastic_update_analysis(dim, nnode, X.reshape(-1).copy(), _f64(C_mat).reshape(-1).copy(),
                                                  int(order), uv.ctypes.data, action.encode(), 1, Ke, Fe, sums)
        if rc:
            raise ValueError("ref_elastic_update_analysis refused the element")
        return Ke.reshape(n, n), Fe, sums.reshape(3, 6)

    def elastic_update(self, X, C_mat, order, action, u=None):
        """The reference's own element driver update(action, u) of
        ElasticityElement3D (X: 8 x 3) or ElasticityElement2D (X: 4 x 2):
        (Ke upper triangle, Fe, integrals of strain, stress, energy (6 each))."""
        X = _f64(X)
        dim, nnode = X.shape[1], X.shape[0]
        n = dim * nnode
        Ke, Fe, sums = np.zeros(n * n), np.zeros(n), np.zeros(18)
        uv = None if u is None else _f64(u).reshape(-1).copy()
        rc = self.lib.ref_elastic_update(dim, nnode, X.reshape(-1).copy(), _f64(C_mat).reshape(-1).copy(), int(order),
                                         None if uv is None else uv.ctypes.data, action.encode(), Ke, Fe, sums)
        if rc:
            raise ValueError("ref_elastic_update refused the element")
        return Ke.reshape(n, n), Fe, sums.reshape(3, 6)

    def heat_update(self, X, k3, cap, order, action="KM", u=None):
        """The reference's own diffusion driver update(action, u) of
        HeatTransferElement3Dtransient (X: 8 x 3) or ...2Dtransient (X: 4 x 2):
        (K, M) upper triangles."""
        X = _f64(X)
        n = X.shape[0]
        K, M = np.zeros(n * n), np.zeros(n * n)
        uv = None if u is None else _f64(u).reshape(-1).copy()
        k = np.zeros(3)
        k[:len(k3)] = k3
        rc = self.lib.ref_heat_update(X.shape[1], n, X.reshape(-1).copy(), k, float(cap), int(order),
                                      None if uv is None else uv.ctypes.data, action.encode(), K, M)
        if rc:
            raise ValueError("ref_heat_update refused the element")
        return K.reshape(n, n), M.reshape(n, n)

    def elastic_vol_avg(self, X, C_mat, order, u):
        """getVolAvgValues: [volume, stress integral (6), strain integral (6),
        SED (3)]."""
        X = _f64(X)
        out = np.zeros(16)
        rc = self.lib.ref_elastic_vol_avg(X.shape[1], X.shape[0], X.reshape(-1).copy(), _f64(C_mat).reshape(-1).copy(),
                                          int(order), _f64(u).reshape(-1).copy(), out)
        if rc:
            raise ValueError("ref_elastic_vol_avg refused the element")
        return out

    def elastic_quad4_ke(self, xy, C9, order):
        """Quad4 plane stiffness (nel x 8 x 8 upper triangles) through the
        reference's Gauss rule, shape functions and ElasticityElement2D."""
        xy = _f64(xy).reshape(-1, 8)
        nel = xy.shape[0]
        Ke = np.zeros(nel * 64)
        if self.lib.ref_elastic_quad4_ke(nel, xy.reshape(-1).copy(), _f64(C9).reshape(-1).copy(), int(order), Ke):
            raise ValueError("ref_elastic_quad4_ke: non-positive Jacobian")
        return Ke.reshape(nel, 8, 8)

    def heat_hex8_k(self, xyz, k3, order):
        """Hex8 conductivity matrices (nel x 8 x 8 upper triangles) through the
        reference's HeatTransferElement3Dtransient::addToKe."""
        xyz = _f64(xyz).reshape(-1, 24)
        nel = xyz.shape[0]
        K = np.zeros(nel * 64)
        if self.lib.ref_heat_hex8_k(nel, xyz.reshape(-1).copy(), _f64(k3).reshape(-1).copy(), int(order), K):
            raise ValueError("ref_heat_hex8_k: non-positive Jacobian")
        return K.reshape(nel, 8, 8)

    def heat_hex8_step_terms(self, xyz, k3, cap, order, u_e, a1, a2, dt):
        """Per hex8 diffusion element (xyz nel x 8 x 3, k3 nel x 3, cap nel,
        nodal u_e nel x 8): the reference's K, M (addToKe, addToMe) and step
        terms (formK_s, formF_s_new) -> (Mbar nel x 8 x 8, F nel x 8)."""
        xyz = _f64(xyz).reshape(-1, 24)
        nel = xyz.shape[0]
        Mb, F = np.zeros(nel * 64), np.zeros(nel * 8)
        rc = self.lib.ref_heat_hex8_step_terms(nel, xyz.reshape(-1).copy(), _f64(k3).reshape(-1).copy(),
                                               _f64(cap).reshape(-1).copy(), int(order),
                                               _f64(u_e).reshape(-1).copy(), float(a1), float(a2), float(dt), Mb, F)
        if rc:
            raise ValueError("ref_heat_hex8_step_terms: non-positive Jacobian")
        return Mb.reshape(nel, 8, 8), F.reshape(nel, 8)

    def print_lower(self, path, fmt, row_ptr, col, val):
        """The reference's printMatrixAddressFormat (fmt 1), ...Upper (2) or
        printCompressedRowFormat (3) of a lower triangle."""
        rc = self.lib.ref_print_lower(str(path).encode(), int(fmt), len(row_ptr) - 1,
                                      np.ascontiguousarray(row_ptr, dtype=np.int64),
                                      np.ascontiguousarray(col, dtype=np.int32),
                                      np.ascontiguousarray(val, dtype=np.float64))
        if rc:
            raise ValueError("ref_print_lower failed")

    def write_csr(self, path, binary, row_ptr, col, val):
        """The reference's writeCSRMatrixIn{ASCII,Binary}."""
        self.lib.ref_write_csr(str(path).encode(), int(binary), len(row_ptr) - 1, len(col),
                               np.ascontiguousarray(row_ptr, dtype=np.int32), np.ascontiguousarray(col, dtype=np.int32),
                               np.ascontiguousarray(val, dtype=np.float64))

    def read_csr(self, path, binary):
        """The reference's readCSRMatrixIn{ASCII,Binary}: (row_ptr, col, val)."""
        n, nz = C.c_int(0), C.c_int(0)
        self.lib.ref_read_csr(str(path).encode(), int(binary), C.byref(n), C.byref(nz), None, None, None)
        ia = np.zeros(n.value + 1, dtype=np.int32)
        ja = np.zeros(nz.value, dtype=np.int32)
        a = np.zeros(nz.value)
        self.lib.ref_read_csr(str(path).encode(), int(binary), C.byref(n), C.byref(nz), ia.ctypes.data,
                              ja.ctypes.data, a.ctypes.data)
        return ia, ja, a

    def sparse_solve_file(self, path, rhs, eps, maxit=1000000):
        """The reference's SymmetricSparseMatrix::readMatrixAddressFormat +
        solve on a lower-triangle address-format file; returns (x, iterations)."""
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        x = np.zeros_like(rhs)
        it = C.c_int(0)
        rc = self.lib.ref_sparse_solve_file(str(path).encode(), rhs, float(eps), int(maxit), x, C.byref(it))
        if rc:
            raise ValueError("not a lower-triangle address-format file")
        return x, it.value
