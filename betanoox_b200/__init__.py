"""B200-native element assembly + PCG path for BETA (kaushik-d/BetaNoOx).

The compute path is the C ABI in include/beta_gpu.h, implemented by
hand-written sm_100a kernels in csrc/ and built in-tree into
_lib/libbeta_gpu.so.  This package adds a thin Python view of that ABI
(:class:`Solver`) mirroring BETA's Equations / assembler calls, plus seeded
workload generators.  Nothing here computes on the CPU in place of the GPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import BetaGpuError, SolveOpts, SolveStats

__all__ = ["Solver", "Batch", "Server", "surface_flux_load", "parse_element_groups", "write_lower", "read_lower", "read_mesh", "write_mesh", "SolveOpts", "SolveStats", "BetaGpuError", "build", "opts"]


def build(force: bool = False) -> str:
    from .build import build as _b
    return _b(force=force)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def opts(mode=_abi.MODE_MPIR, precond=_abi.PRECOND_BLOCK_JACOBI, stop_rule=_abi.STOP_RB, tol=1e-10,
         maxit=100000, inner_tol=0.01, max_outer=60, use_last_solution=0, check_every=0, profile=False):
    return SolveOpts(mode, precond, stop_rule, maxit, tol, inner_tol, max_outer, use_last_solution, check_every,
                     1 if profile else 0)


class Solver:
    """One device-resident finite-element system (a beta_gpu context).

    Mirrors the BETA sequence: mesh/material/boundary upload (ReadMesh,
    SetElementProperty, loads applyTo), build_pattern (allocateEquationsMatrix),
    assemble (assembler->assembleK), solve (Equations::solve).
    """

    def __init__(self, device: int = 0):
        self.lib = _abi.load()
        h = C.c_void_p()
        st = self.lib.beta_gpu_create(C.byref(h), device)
        if st != _abi.OK:
            raise BetaGpuError(st, "beta_gpu_create failed (no usable CUDA device?)")
        self.h = h
        self.model = None

    def close(self):
        if getattr(self, "h", None):
            self.lib.beta_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st, what=""):
        if st != _abi.OK:
            msg = self.lib.beta_gpu_last_error(self.h)
            raise BetaGpuError(st, f"{what}: {msg.decode() if msg else ''}")
        return st

    # -- upload -------------------------------------------------------------
    def load_model(self, m, params=None, elem_group=None):
        self.model = m
        xyz = np.ascontiguousarray(m.xyz, dtype=np.float64)
        conn = np.ascontiguousarray(m.conn, dtype=np.int32)
        fd = np.ascontiguousarray(m.first_dof, dtype=np.int32)
        self._check(self.lib.beta_gpu_mesh_upload(self.h, m.kind, m.ndim, m.nnode, _ptr(xyz), m.nelem, m.nnpe,
                                                  _ptr(conn), _ptr(fd), m.ndpn, m.order), "mesh_upload")
        self.load_materials(m.params if params is None else params, elem_group)
        self.set_bc(m.restrained, m.prescribed, m.load)

    def load_materials(self, params, elem_group=None):
        """Material parameters per group (one group per element without
        elem_group); the assembled matrices are rebuilt at their next use."""
        p = np.ascontiguousarray(params, dtype=np.float64)
        eg = None if elem_group is None else np.ascontiguousarray(elem_group, dtype=np.int32)
        self._check(self.lib.beta_gpu_materials_upload(self.h, p.shape[0], p.shape[1], _ptr(p), _ptr(eg)),
                    "materials_upload")

    def set_bc(self, restrained, prescribed, load):
        r = np.ascontiguousarray(restrained, dtype=np.uint8)
        p = np.ascontiguousarray(prescribed, dtype=np.float64)
        ld = np.ascontiguousarray(load, dtype=np.float64)
        self._check(self.lib.beta_gpu_bc_upload(self.h, _ptr(r), _ptr(p), _ptr(ld)), "bc_upload")

    def build_pattern(self):
        nnz = C.c_longlong(0)
        self._check(self.lib.beta_gpu_build_pattern(self.h, C.byref(nnz)), "build_pattern")
        self.nnz_lower = int(nnz.value)
        return self.nnz_lower

    def set_block_runs(self, run):
        """Column runs of the FP32 block matrix: 3 (default) stores one column
        index per run of up to three consecutive node columns where that
        shrinks the matrix by 5 % or more, 1 one index per block.  Applies at
        the next build_pattern."""
        self._check(self.lib.beta_gpu_set_block_runs(self.h, int(run)), "set_block_runs")

    def set_operator_cache(self, on):
        """Keep the FP64 element matrices of a hex8 diffusion mesh on the
        device for the FP64 operator (True, the default) or integrate them at
        every use (False)."""
        self._check(self.lib.beta_gpu_set_operator_cache(self.h, 1 if on else 0), "set_operator_cache")

    def block_layout(self):
        """(run length, value chunks, column indices read, bytes, compact) of
        the FP32 block matrix as built."""
        out = (C.c_longlong * 5)()
        self._check(self.lib.beta_gpu_block_layout(self.h, out, 5), "block_layout")
        return tuple(int(v) for v in out)

    def pattern_lower(self):
        n = self.model.ndof
        rp = np.zeros(n + 1, dtype=np.int64)
        col = np.zeros(self.nnz_lower, dtype=np.int32)
        self._check(self.lib.beta_gpu_pattern_lower(self.h, _ptr(rp), _ptr(col)), "pattern_lower")
        return rp, col

    def assemble(self, precision=_abi.FP32, what=_abi.ASM_K, dt=0.0, alpha=1.0):
        self._check(self.lib.beta_gpu_assemble(self.h, what, precision, dt, alpha), "assemble")

    def element_outputs(self, u=None):
        """Per element [volume, int stress dV, int strain dV, strain energy]
        (getVolAvgValues) and their sums over the mesh; u: displacements or
        None for the last solution."""
        m = self.model
        ns = 6 if m.kind == _abi.HEX8_ELASTIC else 3
        per = np.zeros((m.nelem, 2 * ns + 2))
        tot = np.zeros(2 * ns + 2)
        uu = None if u is None else np.ascontiguousarray(u, dtype=np.float64)
        self._check(self.lib.beta_gpu_element_outputs(self.h, _ptr(uu), _ptr(per), _ptr(tot)), "element_outputs")
        return per, tot

    def export_matrix(self, path, fmt, precision=_abi.FP64):
        """Writes the assembled matrix in one of BETA's exchange formats."""
        self._check(self.lib.beta_gpu_export_matrix(self.h, precision, int(fmt), str(path).encode()), "export_matrix")

    def lower_values(self, precision):
        vals = np.zeros(self.nnz_lower)
        pl = np.zeros(self.model.ndof)
        self._check(self.lib.beta_gpu_matrix_lower_values(self.h, precision, _ptr(vals), _ptr(pl)), "lower_values")
        return vals, pl

    def set_zero_diagonal(self, value):
        """ReplaceZeroDiagonal: 0 refuses a zero global diagonal at the solve;
        another value replaces every zero diagonal by it."""
        self._check(self.lib.beta_gpu_set_zero_diagonal(self.h, float(value)), "set_zero_diagonal")

    def solve(self, o=None, raise_on_error=True):
        o = o or opts()
        st = SolveStats()
        rc = self.lib.beta_gpu_solve(self.h, C.byref(o), C.byref(st))
        if raise_on_error:
            self._check(rc, "solve")
        return rc, st

    def download(self):
        u = np.zeros(self.model.ndof)
        self._check(self.lib.beta_gpu_download(self.h, _ptr(u)), "download")
        return u

    def matvec(self, x, precision=_abi.FP64):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros_like(x)
        self._check(self.lib.beta_gpu_matvec(self.h, precision, _ptr(x), _ptr(y)), "matvec")
        return y

    def internal_force(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        f = np.zeros_like(u)
        self._check(self.lib.beta_gpu_internal_force(self.h, _ptr(u), _ptr(f)), "internal_force")
        return f

    # -- transient diffusion -------------------------------------------------
    def set_solution(self, u):
        """The current solution (a Newton loop's starting point, the tangent's displacement)."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        self._check(self.lib.beta_gpu_set_solution(self.h, _ptr(u)), "set_solution")

    def internal_force_nonlinear(self, u):
        """The geometric-nonlinear internal force f(u) (hex8 elasticity)."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        f = np.zeros_like(u)
        self._check(self.lib.beta_gpu_internal_force_nonlinear(self.h, _ptr(u), _ptr(f)), "internal_force_nonlinear")
        return f

    def newton(self, solve=None, max_residual=1e-10, max_newton=400, use_last_solution=False,
               raise_on_error=True):
        """BasicModel::iterate with the geometric-nonlinear hex8 element:
        returns (rc, stats, history of max |R| per iteration)."""
        o = _abi.NewtonOpts()
        o.max_residual = max_residual
        o.max_newton = max_newton
        o.use_last_solution = int(bool(use_last_solution))
        o.solve = solve or opts(mode=_abi.MODE_FP64, stop_rule=_abi.STOP_REF, tol=1e-10, maxit=100000)
        st = _abi.NewtonStats()
        hist = np.zeros(max_newton + 1)
        rc = self.lib.beta_gpu_newton(self.h, C.byref(o), C.byref(st), _ptr(hist))
        if raise_on_error and rc not in (_abi.OK,):
            self._check(rc, "newton")
        return rc, st, hist[:st.iterations + 1]

    def heat_set_state(self, u0):
        u0 = np.ascontiguousarray(u0, dtype=np.float64)
        self._check(self.lib.beta_gpu_heat_set_state(self.h, _ptr(u0)), "heat_set_state")

    def heat_run(self, dt, nsteps, o=None, alpha=1.0):
        o = o or opts()
        st = SolveStats()
        tot = C.c_int(0)
        self._check(self.lib.beta_gpu_heat_run(self.h, dt, alpha, nsteps, C.byref(o), C.byref(st), C.byref(tot)),
                    "heat_run")
        return st, int(tot.value)

    def heat_get_state(self):
        u = np.zeros(self.model.ndof)
        self._check(self.lib.beta_gpu_heat_get_state(self.h, _ptr(u)), "heat_get_state")
        return u


def parse_element_groups(text, nelem, init=-1):
    """Element -> material group map from the body of a setElementMaterial
    block of a BETA input deck (lines "first last increment group" or
    "all group", ended by "end"); elements not named keep `init`."""
    lib = _abi.load()
    g = np.full(int(nelem), int(init), dtype=np.int32)
    n = C.c_int(0)
    st = lib.beta_gpu_parse_element_groups(text.encode() if isinstance(text, str) else bytes(text), int(nelem),
                                           _ptr(g), C.byref(n))
    if st != _abi.OK:
        raise BetaGpuError(st, "parse_element_groups: malformed setElementMaterial block")
    return g


def surface_flux_load(face_conn, xyz, nodal_flux, first_dof, ndof, load=None):
    """Consistent nodal loads of a nodal surface flux (SurfaceLoad::applyTo):
    face_conn (nface x 4, 6 or 8 node ids), xyz (nnode x 3), nodal_flux
    (nnode), first_dof (nnode).  The loads are added to `load` (a new zero
    vector of ndof when None), which is returned."""
    lib = _abi.load()
    fc = np.ascontiguousarray(face_conn, dtype=np.int32)
    if fc.ndim != 2:
        raise ValueError("face_conn must be nface x nodes_per_face")
    x = np.ascontiguousarray(xyz, dtype=np.float64)
    q = np.ascontiguousarray(nodal_flux, dtype=np.float64)
    fd = np.ascontiguousarray(first_dof, dtype=np.int32)
    out = np.zeros(ndof) if load is None else load
    if out.dtype != np.float64 or not out.flags.c_contiguous or out.shape != (ndof,):
        raise ValueError("load must be a contiguous float64 vector of ndof")
    if x.shape != (q.shape[0], 3) or fd.shape != q.shape:
        raise ValueError("xyz must be nnode x 3, nodal_flux and first_dof nnode")
    st = lib.beta_gpu_surface_flux_load(fc.shape[0], fc.shape[1], _ptr(fc), q.shape[0], _ptr(x), _ptr(q), _ptr(fd),
                                        int(ndof), _ptr(out))
    if st != _abi.OK:
        raise BetaGpuError(st, "surface_flux_load")
    return out


def write_lower(path, fmt, row_ptr, col, val):
    """Writes a lower triangle in one of BETA's exchange formats (_abi.FMT_*)."""
    lib = _abi.load()
    rp = np.ascontiguousarray(row_ptr, dtype=np.int64)
    c = np.ascontiguousarray(col, dtype=np.int32)
    v = np.ascontiguousarray(val, dtype=np.float64)
    st = lib.beta_gpu_write_lower(str(path).encode(), int(fmt), len(rp) - 1, _ptr(rp), _ptr(c), _ptr(v))
    if st != _abi.OK:
        raise BetaGpuError(st, f"write_lower {path}")


def read_lower(path, fmt):
    """Reads a lower triangle written in one of BETA's exchange formats: (row_ptr, col, val)."""
    lib = _abi.load()
    n, nnz = C.c_int(0), C.c_longlong(0)
    st = lib.beta_gpu_read_lower(str(path).encode(), int(fmt), C.byref(n), C.byref(nnz), None, None, None)
    if st != _abi.OK:
        raise BetaGpuError(st, f"read_lower {path}")
    rp = np.zeros(n.value + 1, np.int64)
    col = np.zeros(nnz.value, np.int32)
    val = np.zeros(nnz.value)
    st = lib.beta_gpu_read_lower(str(path).encode(), int(fmt), C.byref(n), C.byref(nnz), _ptr(rp), _ptr(col),
                                 _ptr(val))
    if st != _abi.OK:
        raise BetaGpuError(st, f"read_lower {path}")
    return rp, col, val


def read_mesh(path, binary=False):
    """Reads a BETA mesh file: (xyz[nnode, ndim], conn[nelem, nnpe]) with
    0-based node indices in BETA's local order."""
    lib = _abi.load()
    nd, nn, ne, npe = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    args = (str(path).encode(), int(bool(binary)), C.byref(nd), C.byref(nn), C.byref(ne), C.byref(npe))
    st = lib.beta_gpu_read_mesh(*args, None, None)
    if st != _abi.OK:
        raise BetaGpuError(st, f"read_mesh {path}")
    xyz = np.zeros((nn.value, nd.value))
    conn = np.zeros((ne.value, npe.value), np.int32)
    st = lib.beta_gpu_read_mesh(*args, _ptr(xyz), _ptr(conn))
    if st != _abi.OK:
        raise BetaGpuError(st, f"read_mesh {path}")
    return xyz, conn


def write_mesh(path, xyz, conn, binary=False, first_number=1):
    """Writes a mesh in BETA's mesh-file layout (nodes and elements numbered from first_number)."""
    lib = _abi.load()
    x = np.ascontiguousarray(xyz, dtype=np.float64)
    c = np.ascontiguousarray(conn, dtype=np.int32)
    st = lib.beta_gpu_write_mesh(str(path).encode(), int(bool(binary)), x.shape[1], x.shape[0], _ptr(x), c.shape[0],
                                 c.shape[1], _ptr(c), int(first_number))
    if st != _abi.OK:
        raise BetaGpuError(st, f"write_mesh {path}")


class Batch:
    """Many independent systems solved in one persistent launch (beta_gpu_batch)."""

    def __init__(self, device: int = 0, hbm_budget: int = 8 << 30, max_systems: int = 4096):
        self.lib = _abi.load()
        h = C.c_void_p()
        st = self.lib.beta_gpu_batch_create(C.byref(h), device, int(hbm_budget), int(max_systems))
        if st != _abi.OK:
            raise BetaGpuError(st, "beta_gpu_batch_create failed")
        self.h = h
        self.models = {}

    def close(self):
        if getattr(self, "h", None):
            self.lib.beta_gpu_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _err(self, st, what):
        msg = self.lib.beta_gpu_batch_last_error(self.h)
        return BetaGpuError(st, f"{what}: {msg.decode() if msg else ''}")

    def add(self, m, raise_on_reject=True):
        """Returns the system id, or None when the pool has no room (REJECTED)."""
        xyz = np.ascontiguousarray(m.xyz, dtype=np.float64)
        conn = np.ascontiguousarray(m.conn, dtype=np.int32)
        fd = np.ascontiguousarray(m.first_dof, dtype=np.int32)
        p = np.ascontiguousarray(m.params, dtype=np.float64)
        r = np.ascontiguousarray(m.restrained, dtype=np.uint8)
        pr = np.ascontiguousarray(m.prescribed, dtype=np.float64)
        ld = np.ascontiguousarray(m.load, dtype=np.float64)
        sid = C.c_int(-1)
        st = self.lib.beta_gpu_batch_add(self.h, m.kind, m.ndim, m.nnode, _ptr(xyz), m.nelem, m.nnpe, _ptr(conn),
                                         _ptr(fd), m.ndpn, m.order, p.shape[0], p.shape[1], _ptr(p), None, _ptr(r),
                                         _ptr(pr), _ptr(ld), C.byref(sid))
        if st == _abi.REJECTED and not raise_on_reject:
            return None
        if st != _abi.OK:
            raise self._err(st, "batch_add")
        self.models[sid.value] = m
        return sid.value

    def add_many(self, models, host_threads=0):
        """Adds models with their structures built on host_threads host
        threads (0 = all cores); returns the ids (None where REJECTED)."""
        keep = []
        arr = (_abi.System * len(models))()
        for k, m in enumerate(models):
            a = dict(xyz=np.ascontiguousarray(m.xyz, dtype=np.float64),
                     conn=np.ascontiguousarray(m.conn, dtype=np.int32),
                     first_dof=np.ascontiguousarray(m.first_dof, dtype=np.int32),
                     group_params=np.ascontiguousarray(m.params, dtype=np.float64),
                     restrained=np.ascontiguousarray(m.restrained, dtype=np.uint8),
                     prescribed=np.ascontiguousarray(m.prescribed, dtype=np.float64),
                     load=np.ascontiguousarray(m.load, dtype=np.float64))
            keep.append(a)
            s = arr[k]
            s.kind, s.ndim, s.nnode, s.nelem, s.nnpe = m.kind, m.ndim, m.nnode, m.nelem, m.nnpe
            s.ndof_per_node, s.integration_order = m.ndpn, m.order
            s.ngroups, s.nparams = a["group_params"].shape
            for f, v in a.items():
                setattr(s, f, v.ctypes.data)
        ids = (C.c_int * max(1, len(models)))()
        st = self.lib.beta_gpu_batch_add_many(self.h, len(models), arr, int(host_threads), ids)
        out = []
        for k, m in enumerate(models):
            if ids[k] >= 0:
                self.models[ids[k]] = m
                out.append(ids[k])
            elif -ids[k] == _abi.REJECTED:
                out.append(None)
            else:
                raise self._err(-ids[k], f"batch_add_many (system {k})")
        del keep
        return out

    def run(self, o=None, iters_per_launch=0):
        """One persistent launch; returns the number of unfinished systems."""
        o = o or opts()
        left = C.c_int(0)
        st = self.lib.beta_gpu_batch_run(self.h, C.byref(o), int(iters_per_launch), C.byref(left))
        if st != _abi.OK:
            raise self._err(st, "batch_run")
        return left.value

    def result(self, sid, with_u=True):
        st = SolveStats()
        u = np.zeros(self.models[sid].ndof) if with_u else None
        rc = self.lib.beta_gpu_batch_result(self.h, sid, _ptr(u), C.byref(st))
        return rc, u, st

    def remove(self, sid):
        st = self.lib.beta_gpu_batch_remove(self.h, sid)
        if st != _abi.OK:
            raise self._err(st, "batch_remove")
        self.models.pop(sid, None)

    def tune(self, threads, gang_boost=4):
        """threads per CTA (256/512/1024); a system gets about gang_boost x its
        share of the batch's CTAs as one gang when that is >= 2 (0: no gangs)."""
        st = self.lib.beta_gpu_batch_tune(self.h, threads, gang_boost)
        if st != _abi.OK:
            raise self._err(st, "batch_tune")

    def autotune(self, o=None, budget=40):
        """budget iterations per system for each launch shape; 0 = complete solves."""
        o = o or opts()
        t, c = C.c_int(0), C.c_int(0)
        st = self.lib.beta_gpu_batch_autotune(self.h, C.byref(o), budget, C.byref(t), C.byref(c))
        if st != _abi.OK:
            raise self._err(st, "batch_autotune")
        return t.value, c.value

    def set_switch(self, iters_per_cycle):
        """FP32 cycles longer than this switch a system to FP64 matrix-free PCG (0: never)."""
        st = self.lib.beta_gpu_batch_set_switch(self.h, int(iters_per_cycle))
        if st != _abi.OK:
            raise self._err(st, "batch_set_switch")

    def set_slice(self, slice_us):
        """Time slice of a launch in microseconds (0: off): systems stop after
        the iteration in which it ends; results do not change."""
        st = self.lib.beta_gpu_batch_set_slice(self.h, int(slice_us))
        if st != _abi.OK:
            raise self._err(st, "batch_set_slice")

    def reset(self):
        """Marks every system unsolved (the next run re-assembles and re-solves)."""
        st = self.lib.beta_gpu_batch_reset(self.h)
        if st != _abi.OK:
            raise self._err(st, "batch_reset")

    INFO = ["live", "used", "pool", "launches", "h2d", "d2h", "last_launch_ns", "gangs", "gang_ctas", "threads",
            "gang_boost", "sys_busy_ns", "sys_setup_ns", "sys_repl_ns", "iterations"]

    def info(self):
        a = (C.c_longlong * len(self.INFO))()
        self.lib.beta_gpu_batch_info(self.h, a, len(self.INFO))
        return dict(zip(self.INFO, list(a)))


class Server:
    """Continuous-batching solve server (beta_gpu_server): submit systems at any
    time; a native worker thread admits them into an HBM pool, solves them in
    bounded persistent launches alongside whatever else is in flight, and
    retires each as soon as it converges."""

    STATS = ["submitted", "done", "rejected", "failed", "cancelled", "queued", "running", "launches",
             "pool_used", "pool_bytes", "busy_us", "h2d", "d2h", "sys_busy_ns", "sys_setup_ns", "sys_repl_ns",
             "iterations"]

    def __init__(self, device: int = 0, hbm_budget: int = 8 << 30, max_systems: int = 4096, o=None,
                 iters_per_launch: int = 200, threads: int = 0, gang_boost: int = -1, slice_us: int = 0):
        self.lib = _abi.load()
        self.o = o or opts()
        h = C.c_void_p()
        st = self.lib.beta_gpu_server_create(C.byref(h), device, int(hbm_budget), int(max_systems),
                                             C.byref(self.o), int(iters_per_launch), int(threads), int(gang_boost))
        if st != _abi.OK:
            raise BetaGpuError(st, "beta_gpu_server_create failed")
        self.h = h
        if slice_us:
            st = self.lib.beta_gpu_server_set_slice(h, int(slice_us))
            if st != _abi.OK:
                self.close()
                raise BetaGpuError(st, "beta_gpu_server_set_slice failed")

    def close(self):
        if getattr(self, "h", None):
            self.lib.beta_gpu_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, m):
        """Queues model m; returns the request id (input errors raise at once)."""
        xyz = np.ascontiguousarray(m.xyz, dtype=np.float64)
        conn = np.ascontiguousarray(m.conn, dtype=np.int32)
        fd = np.ascontiguousarray(m.first_dof, dtype=np.int32)
        p = np.ascontiguousarray(m.params, dtype=np.float64)
        r = np.ascontiguousarray(m.restrained, dtype=np.uint8)
        pr = np.ascontiguousarray(m.prescribed, dtype=np.float64)
        ld = np.ascontiguousarray(m.load, dtype=np.float64)
        rid = C.c_longlong(0)
        st = self.lib.beta_gpu_server_submit(self.h, m.kind, m.ndim, m.nnode, _ptr(xyz), m.nelem, m.nnpe, _ptr(conn),
                                             _ptr(fd), m.ndpn, m.order, p.shape[0], p.shape[1], _ptr(p), None,
                                             _ptr(r), _ptr(pr), _ptr(ld), C.byref(rid))
        if st != _abi.OK:
            msg = self.lib.beta_gpu_server_last_error(self.h)
            raise BetaGpuError(st, f"server_submit: {msg.decode() if msg else ''}")
        return rid.value

    def poll(self, rid, wait_ms=0, release=False):
        """Returns (state, u or None, stats, latency_ms)."""
        state, nd = C.c_int(0), C.c_int(0)
        st = SolveStats()
        lat = C.c_double(-1.0)
        rc = self.lib.beta_gpu_server_poll(self.h, rid, 0, C.byref(state), C.byref(nd), None, None, None, 0)
        if rc != _abi.OK:
            raise BetaGpuError(rc, f"server_poll: unknown request {rid}")
        u = np.zeros(nd.value)
        rc = self.lib.beta_gpu_server_poll(self.h, rid, int(wait_ms), C.byref(state), None, _ptr(u), C.byref(st),
                                           C.byref(lat), int(bool(release)))
        if rc != _abi.OK:
            raise BetaGpuError(rc, f"server_poll: unknown request {rid}")
        return state.value, (u if state.value == _abi.REQ_DONE else None), st, lat.value

    def wait(self, rid, timeout_s=120.0, release=True):
        """Blocks until the request is final; returns (state, u, stats, latency_ms)."""
        import time
        end = time.monotonic() + timeout_s
        while True:
            left = max(1, int((end - time.monotonic()) * 1000))
            state, u, st, lat = self.poll(rid, wait_ms=min(left, 1000), release=False)
            if state >= _abi.REQ_DONE:
                if release:
                    self.poll(rid, release=True)
                return state, u, st, lat
            if time.monotonic() > end:
                raise TimeoutError(f"request {rid} not finished after {timeout_s} s")

    def cancel(self, rid):
        rc = self.lib.beta_gpu_server_cancel(self.h, rid)
        if rc != _abi.OK:
            raise BetaGpuError(rc, f"server_cancel: unknown request {rid}")

    def stats(self):
        a = (C.c_longlong * len(self.STATS))()
        self.lib.beta_gpu_server_stats(self.h, a, len(self.STATS))
        return dict(zip(self.STATS, list(a)))
