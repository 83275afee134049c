"""Benchmark of the BETA assembly + PCG path on B200.

Default workload (N=1): 3D hex8 linear elasticity on a structured
100x100x100 cube (1,030,301 nodes, 3,090,903 dofs), 2x2x2 Gauss, per-element
E = 1e4*exp(N(0,0.5^2)), nu ~ U[0.20,0.35], z=0 clamped, pressure 1.0 on z=1.
One step = FP32 assembly + mixed-precision refinement solve (FP32 block-Jacobi
inner PCG, FP64 matrix-free outer residual and update) to
||b - A u||/||b|| <= tol, inputs resident in HBM.  The plain FP64 GPU
Jacobi-PCG is measured on the same workload for the mixed/plain ratio.

Multi-GPU (torchrun): every rank solves its own replica (the path does not
shard: one system per GPU); value = total dofs solved / max-over-ranks time.

--config batch: 512 two-phase RVE cubes (n ~ U{8..40}) solved together in one
persistent launch (gangs of CTAs for big systems, single CTAs for small ones,
autotuned launch shape);
one step = reset + assembly + mixed-precision solve of all 512.
--config heat: transient diffusion on a 256x256x64 hex8 slab, 100 backward-Euler
steps (each assembles C/dt + K in FP32 and solves it).
--config serve: a Poisson stream of requests (quad4 / hex8 elasticity / hex8
diffusion, log-uniform 1e3-5e5 dofs) through the continuous-batching server at
80% of its measured capacity; reports throughput and p50/p99 latency.

--impl reference: the reference's CPU path on a bounded sample of the same
workload, extrapolated to the full solve (see cpu_baseline.sample in the
output).  For the cube this is the reference's own code compiled from its
sources (oracle/_ref: element B/addToKe, Equations pattern and addMatrix,
and the faster of its SymmetricSparseMatrix::solve and two-thread ParCG
solve), with the oracle's all-core port beside it; elsewhere, or without oracle/_ref, the
oracle's port on all host cores.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solved DOFs/s at <=1e-8 rel err, mixed vs plain FP64 GPU PCG; p50/p99 latency"
UNIT = "DOF/s"


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Clocks:
    """Samples SM clock and throttle reasons every 200 ms during the timed
    region through NVML in-process (no nvidia-smi process per sample)."""

    # NVML clocks-event reason bits
    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
               0x4: "sw_power_cap"}

    def __init__(self, gpu):
        self.gpu = gpu
        self.rows = []
        self._stop = threading.Event()
        self._t = None
        self._h = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nv = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(gpu)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
        except Exception as e:  # no NVML: report it, keep timing
            self._err = str(e)
            self.max_mhz = None

    def _run(self):
        nv = self._nv
        while not self._stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                self.rows.append((sm, rs))
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        if self._h is not None:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz,
                    "reasons": [getattr(self, "_err", "no samples")], "samples": 0}
        reasons = set()
        for _, rs in self.rows:
            for bit, nm in self.REASONS.items():
                if rs & bit:
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(r[0] for r in self.rows), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(reasons), "samples": len(self.rows), "source": "nvml"}


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def _traffic(name="spmv_traffic.json"):
    p = os.path.join(ROOT, "profiles", name)
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return None


def make_model(cfg, n):
    from betanoox_b200 import workloads as W
    if cfg == "cube":
        return W.cube_hex8(n)
    raise SystemExit(f"unknown config {cfg}")


def _pinned_copy(a):
    import torch
    t = torch.empty(a.shape, dtype={np.float64: torch.float64, np.int32: torch.int32,
                                     np.uint8: torch.uint8}[a.dtype.type], pin_memory=True)
    t.numpy()[...] = a
    return t.numpy()


def _phase_shares(d, d0=None):
    """Shares of the systems' group device time (kernel timers): setup
    (assembly, factors, first residual), reliable updates (FP64 residual
    replacements) and inner iterations."""
    g = lambda k: d[k] - (d0[k] if d0 else 0)
    busy = g("sys_busy_ns")
    if busy <= 0:
        return None
    setup, repl = g("sys_setup_ns"), g("sys_repl_ns")
    return {"setup": setup / busy, "reliable_updates": repl / busy, "iterations": (busy - setup - repl) / busy,
            "group_s": busy / 1e9}


def spmv_algorithmic_bytes(nblk, nnode, nd, ncols=None):
    """Per launch of the FP32 node-block SpMV: the nd*nd FP32 values of every
    non-zero block once, the layout's 4-byte column indices once (ncols: one
    per block, or one per run of consecutive node columns as the layout was
    built, padding lanes included), the input vector once and the output
    vector once (nd FP32 per node)."""
    return nblk * nd * nd * 4 + 4 * (nblk if ncols is None else ncols) + 2 * nnode * nd * 4


def _layout_label(layout, nd):
    run = layout[0] if layout else 1
    cols = "one column per block" if run == 1 else f"one column per run of {run} node columns"
    if layout and len(layout) > 4 and layout[4]:
        cols += ", compact"
    return f"k_spmv_dot_b<{nd},{run}> (FP32 node-block sliced ELL, {cols}, + p.Ap)"


def _init_dist(dev, backend="nccl"):
    """One process per GPU under torchrun: a process group with a short
    timeout (ranks that wait for a dead peer end with an error).  The backend
    is NCCL on GPUs; the rank logic is the same with gloo on the host."""
    import torch
    ws, rank, local = _dist()
    if backend == "nccl":
        torch.cuda.set_device(dev)
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        kw = {"device_id": torch.device("cuda", dev)} if backend == "nccl" else {}
        dist.init_process_group(backend, timeout=timedelta(seconds=600), **kw)
    return ws, rank


def _max_over_ranks(v, dev):
    """Max of a per-rank number over all ranks (every rank gets it)."""
    ws, _, _ = _dist()
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    on_gpu = dist.get_backend() == "nccl"
    t = torch.tensor([float(v)], dtype=torch.float64, device=f"cuda:{dev}" if on_gpu else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier():
    import torch
    ws, _, _ = _dist()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
    if torch.cuda.is_available():
        torch.cuda.synchronize()


def whole_job_rate(units_per_rank, seconds, dev=0):
    """Weak-scaling aggregate: every rank processed units_per_rank; the job
    took the slowest rank's time.  Returns (units/s for the whole job, max s)."""
    ws, _, _ = _dist()
    tmax = _max_over_ranks(seconds, dev)
    return ws * units_per_rank / tmax, tmax


def _sub_args(args, which):
    """The arguments of a sub-record run inside the default line: bounded so
    the whole line stays within minutes (stated in each record's config)."""
    a = argparse.Namespace(**vars(args))
    a.skip_cpu = True
    a.steps, a.warmup = args.sub_steps, max(3, args.sub_warmup)
    if which == "batch":
        a.fp64_stride = args.sub_fp64_stride
        a.e2e_steps = 1
    else:
        a.requests = args.sub_requests
        a.capacity_requests = min(args.capacity_requests, args.sub_requests)
        a.serve_pool = min(args.serve_pool, args.sub_requests)
        a.warmup = 1
    return a


_SUB_KEYS = ("value", "unit", "steps", "warmup", "ms_per_step", "config", "latency_ms", "per_step_ms", "fp64_plain",
             "mixed_over_fp64", "capacity_over_fp64", "roofline", "rel_err_vs_fp64_reference", "e2e",
             "gpu_launches", "clocks", "batch", "serve")


def _sub_record(out):
    """The keys of a configuration's own line kept in the default line."""
    if out is None:
        return None
    return {k: out[k] for k in _SUB_KEYS if k in out}


def run_ours(args):
    import torch
    from betanoox_b200 import Solver, _abi, opts

    ws, rank, local = _dist()
    dev = local
    _init_dist(dev)

    m = make_model(args.config, args.n)
    stream = torch.cuda.Stream(device=dev)
    g = Solver(dev)
    g.lib.beta_gpu_set_stream(g.h, C.c_void_p(stream.cuda_stream))
    t0 = time.perf_counter()
    g.load_model(m)
    g.build_pattern()
    t_setup = time.perf_counter() - t0
    lib, h = g.lib, g.h

    tol = args.tol
    o_mp = opts(mode=_abi.MODE_MPIR, precond=_abi.PRECOND_BLOCK_JACOBI, stop_rule=_abi.STOP_RB, tol=tol,
                inner_tol=args.inner_tol, profile=True)
    o_64 = opts(mode=_abi.MODE_FP64, stop_rule=_abi.STOP_RB, tol=tol, profile=True)

    def counters():
        a = (C.c_longlong * 3)()
        lib.beta_gpu_counters(h, a, 3)
        return list(a)

    def step_mp():
        g.assemble(_abi.FP32)
        rc, st = g.solve(o_mp)
        return st

    def step_64():
        g.assemble(_abi.FP64)
        rc, st = g.solve(o_64)
        return st

    barrier = _barrier

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        barrier()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        c0 = counters()
        stats = []
        with torch.cuda.stream(stream):
            for i in range(steps):
                evs[i][0].record(stream)
                stats.append(fn())
                evs[i][1].record(stream)
        barrier()
        c1 = counters()
        ms = [a.elapsed_time(b) for a, b in evs]
        return ms, stats, [c1[k] - c0[k] for k in range(3)]

    # -- mixed precision (headline) --
    with Clocks(dev) as clk:
        ms_mp, st_mp, cnt_mp = timed(step_mp, args.steps, args.warmup)
    u_mp = g.download()
    # -- plain FP64 GPU PCG on the same workload --
    fp64 = None
    if not args.skip_fp64:
        ms_64, st_64, _ = timed(step_64, max(1, min(args.steps, 2)), 1)
        u_64 = g.download()
        fp64 = {"ms": ms_64, "stats": [s.as_dict() for s in st_64], "u": u_64}
    # -- end to end through the C ABI from pinned host buffers --
    e2e = None
    if not args.skip_e2e:
        pm = type(m)(m.name, m.kind, m.ndim, _pinned_copy(m.xyz), _pinned_copy(m.conn), m.ndpn,
                     _pinned_copy(m.params), _pinned_copy(m.restrained), _pinned_copy(m.prescribed),
                     _pinned_copy(m.load), m.order, m.meta)
        u_host = _pinned_copy(np.zeros(m.ndof))
        ge = Solver(dev)
        ge.lib.beta_gpu_set_stream(ge.h, C.c_void_p(stream.cuda_stream))

        e2e_ph = np.zeros(5)

        def e2e_step():
            # wall time per phase (each call returns with its device work done
            # or, for the assembly, queued before the solve that waits for it)
            t = [time.perf_counter()]
            ge.load_model(pm)
            t.append(time.perf_counter())
            ge.build_pattern()
            t.append(time.perf_counter())
            ge.assemble(_abi.FP32)
            t.append(time.perf_counter())
            ge.solve(o_mp)
            t.append(time.perf_counter())
            ge.lib.beta_gpu_download(ge.h, u_host.ctypes.data_as(C.c_void_p))
            t.append(time.perf_counter())
            e2e_ph[:] = np.diff(t)

        def ecnt():
            a = (C.c_longlong * 3)()
            ge.lib.beta_gpu_counters(ge.h, a, 3)
            return list(a)

        e2e_step()
        barrier()
        c0 = ecnt()
        tw = []
        for _ in range(max(1, args.e2e_steps)):
            t1 = time.perf_counter()
            e2e_step()
            torch.cuda.synchronize()
            tw.append(time.perf_counter() - t1)
        c1 = ecnt()
        k = max(1, args.e2e_steps)
        ev, tmed = whole_job_rate(m.ndof, statistics.median(tw), dev)
        e2e = {"value": ev, "unit": UNIT,
               "h2d_bytes_per_step": (c1[1] - c0[1]) // k, "d2h_bytes_per_step": (c1[2] - c0[2]) // k,
               "ms_per_step": 1e3 * tmed,
               "last_step_ms": dict(zip(["mesh_and_bc_upload", "structure", "assembly", "solve", "download"],
                                        [round(1e3 * float(v), 2) for v in e2e_ph]))}
        ge.close()

    # -- reduce timing over ranks --
    value, tot_s = whole_job_rate(m.ndof * args.steps, sum(ms_mp) / 1e3, dev)
    tot_ms = tot_s * 1e3
    ms_step = tot_ms / args.steps
    spmv_ms = statistics.median([s.ms_spmv_avg for s in st_mp])
    layout = g.block_layout()
    g.close()

    # -- the batched and served forms, as sub-records of this line (all ranks) --
    # (serving first: its capacity burst sets the stream's arrival rate, and
    # the batch's long power-capped launches would leave it throttled)
    subs = {}
    if not args.skip_serve:
        subs["serve"] = _sub_record(run_serve(_sub_args(args, "serve"), nested=True))
    if not args.skip_batch:
        subs["batch"] = _sub_record(run_batch(_sub_args(args, "batch"), nested=True))

    out = None
    if rank == 0:
        peak, peak_kind = _peaks()
        alg = spmv_algorithmic_bytes(_nblk(m), m.nnode, m.ndpn, layout[2])
        achieved = alg / (spmv_ms * 1e-3) / 1e9 if spmv_ms > 0 else None
        tr = _traffic()
        kern = _layout_label(layout, m.ndpn)
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None,
                "traffic": (round(tr["traffic_over_algorithmic"] * alg)
                            if tr and tr.get("kernel") == kern.split(" ")[0] else None),
                "kernel": kern,
                "algorithmic_bytes_per_launch": alg, "ms_per_launch": spmv_ms,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback 6.65 TB/s"}
        lat = sorted(ms_mp)
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32 inner / fp64 outer", "data": "synthetic (seeded generator)",
            "config": cube_config(m, args, ws),
            "per_step_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
            "mixed": {"iterations": [s.iterations for s in st_mp], "outer": [s.outer_iterations for s in st_mp],
                      "true_rel_residual": [s.true_rel_residual for s in st_mp], "ms_steps": ms_mp},
            "e2e": e2e, "gpu_launches": cnt_mp[0], "roofline": roof,
            "clocks": clk.summary(), "setup_s": t_setup,
        }
        if fp64:
            v64 = m.ndof / (statistics.median(fp64["ms"]) / 1e3)
            out["fp64_plain"] = {"value": ws * v64, "ms_steps": fp64["ms"],
                                 "iterations": [s["iterations"] for s in fp64["stats"]],
                                 "ms_spmv_avg": [s["ms_spmv_avg"] for s in fp64["stats"]]}
            out["mixed_over_fp64"] = value / (ws * v64)
        out.update(subs)
        # the oracle at full size (host, rank 0, after all GPU timing and
        # collectives): its FP64 solution is the accuracy reference, and its
        # own full solve is the CPU baseline
        truth = None
        if not (args.skip_accuracy and args.skip_cpu):
            truth = oracle_cube_truth(m, args)
        if truth is not None:
            ut = truth["u"]
            nt = np.linalg.norm(ut)
            if not args.skip_accuracy:
                err = {"mixed": float(np.linalg.norm(u_mp - ut) / nt),
                       "oracle": truth["how"], "oracle_iterations": truth["iterations_tight"]}
                if fp64:
                    err["fp64"] = float(np.linalg.norm(fp64["u"] - ut) / nt)
                out["rel_err_vs_oracle"] = err
            if not args.skip_cpu:
                out["cpu_baseline"] = truth["cpu_baseline"]
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return out


def _nblk(m):
    """Stored node-pair blocks of the full symmetric matrix (node graph nnz)."""
    from betanoox_b200 import _abi
    import ctypes as C
    lib = _abi.load()
    # the node graph of a mesh equals the scalar pattern of its ndpn=1 view
    conn = np.ascontiguousarray(m.conn, np.int32)
    fd = np.arange(m.nnode, dtype=np.int32)
    r = np.zeros(m.nnode, np.uint8)
    nnz = C.c_longlong()
    lib.beta_gpu_pattern_lower_host(m.nnode, m.nelem, m.nnpe, 1, conn.ctypes.data, fd.ctypes.data, r.ctypes.data,
                                    C.byref(nnz), None, None)
    return 2 * nnz.value - m.nnode


def cube_config(m, args, ws):
    """The cube workload's config record, the same in both arms."""
    return {"workload": f"hex8 elasticity cube {m.meta['n']}^3, {m.ndof} dofs, lognormal E, "
                        f"2x2x2 Gauss, z=0 clamped, p=1 on z=1",
            "global_batch": ws, "ndof": m.ndof, "nelem": m.nelem, "parallelism": f"replicas x{ws}",
            "tol": args.tol, "stop_rule": "||b-Au||/||b||", "replace_delta": args.inner_tol,
            "l2": "inputs larger than L2 (FP32 matrix ~1 GB per replica)"}


# ---- the oracle at full size (test infrastructure) -------------------------
def oracle_cube_truth(m, args):
    """The oracle on the whole workload, on all host threads, after the GPU
    timing: its FP64 assembly (element matrices on all threads, added in
    element order: bit-identical to the serial restatement of the
    reference's assembly) and its threaded Jacobi-PCG from the same initial
    guess, first to the bench's own stop rule ||r||/||b|| <= tol (a full
    solve, timed: the CPU baseline, nothing extrapolated) and then on to
    ||r||/||b|| <= args.oracle_tol (the accuracy reference)."""
    from oracle import beta_oracle as bo
    th = os.cpu_count() or 1
    s = bo.System(m)
    s.set_bc(m.restrained, m.prescribed, m.load)
    t0 = time.perf_counter()
    s.build_pattern()
    t_struct = time.perf_counter() - t0
    t0 = time.perf_counter()
    rc = s.assemble_threaded(m.params, m.order, th)
    t_asm = time.perf_counter() - t0
    if rc:
        raise RuntimeError(f"oracle assembly failed ({rc})")
    csr = s.csr()
    b = s.rhs()
    del s
    x0 = np.where(np.asarray(m.restrained, bool), m.prescribed, 0.0)
    t0 = time.perf_counter()
    rc, x, st, _ = csr.pcg(b, args.tol, maxit=200000, threads=th, rule=bo.Csr.RULE_RB, x0=x0)
    t_solve = time.perf_counter() - t0
    if rc:
        raise RuntimeError(f"oracle solve failed ({rc})")
    rc, xt, st2, _ = csr.pcg(b, args.oracle_tol, maxit=200000, threads=th, rule=bo.Csr.RULE_RB, x0=x)
    cb = {"value": m.ndof / (t_asm + t_solve), "unit": UNIT, "cores": th, "kind": "port",
          "sample": (f"the whole workload, measured (not extrapolated): the oracle's FP64 assembly of all "
                     f"{m.nelem} elements on {th} threads ({t_asm:.2f} s) + its threaded Jacobi-PCG from zero to "
                     f"||r||/||b|| <= {args.tol:g}, {st.iterations} iterations ({t_solve:.1f} s); the structure "
                     f"({t_struct:.2f} s) is built once, untimed, as on the GPU"),
          "seconds": t_asm + t_solve, "iterations": st.iterations}
    return {"u": xt, "cpu_baseline": cb, "iterations_tight": st.iterations + st2.iterations,
            "how": (f"the oracle's FP64 solution: its own assembly, threaded Jacobi-PCG to ||r||/||b|| <= "
                    f"{args.oracle_tol:g}")}


# ---- the reference arm: the reference's own code (oracle/_ref) ---------------
def _eps_after(trace, k, margin=1e-6):
    """A stop tolerance under which the reference rule's quantity (trace[i]
    after iteration i+1) first falls at iteration k' >= k: the smallest such
    k' whose value lies below every earlier one by the margin.  Returns
    (k', eps) or None."""
    for kk in range(max(1, k), len(trace) + 1):
        v = trace[kk - 1] * (1.0 + margin)
        if all(trace[i] > v for i in range(kk - 1)):
            return kk, v
    return None


def reference_cube_setup(m, args):
    """The whole workload built once by the reference's own code compiled
    from its sources (oracle/_ref): per element its Gauss rule, shape
    functions and ElasticityElement3D B / addToKe (serially, as
    SerialAssembler, the reference's default), Equations
    specifyNonZeroLocation / allocate and addMatrix with the restraint
    elimination, addLoadToEqn; storage ParCGMatrix (its two-thread OpenMP
    solver) or SymmetricSparseMatrix (serial).  The element matrices and the
    scatter are timed in full; the structure is timed apart (built once per
    analysis by the reference, as it is on the GPU).

    The full solve's iteration count to the bench's stop rule
    ||r||/||b|| <= tol comes from the oracle's threaded Jacobi-PCG on the
    reference's own assembled matrix and right-hand side (the same
    recurrence as the reference's solver, step for step); its trace of the
    reference rule sqrt(r.r/x.x) gives the tolerances at which the
    reference's solve stops after a chosen number of iterations."""
    from oracle import beta_oracle as bo
    th = os.cpu_count() or 1
    leaf = bo.RefLeaf()
    Cs = bo.cmat_ortho3d_many(m.params)  # the materials as read: one per element, untimed
    nd = m.nnpe * m.ndpn
    maps = np.ascontiguousarray(
        (m.first_dof[m.conn][:, :, None] + np.arange(m.ndpn)[None, None, :]).reshape(m.nelem, nd), np.int32)
    rs = bo.RefSystem(m.ndof, m.restrained, m.prescribed, parcg=args.ref_solver == "parcg")
    t0 = time.perf_counter()
    rs.pattern(maps)
    rs.allocate()
    t_struct = time.perf_counter() - t0
    t_el = t_add = 0.0
    for e0 in range(0, m.nelem, 32768):
        e1 = min(m.nelem, e0 + 32768)
        xe = np.ascontiguousarray(m.xyz[m.conn[e0:e1]])
        t0 = time.perf_counter()
        Ke = leaf.elastic_hex8_ke(xe, Cs[e0:e1], m.order)
        t_el += time.perf_counter() - t0
        t0 = time.perf_counter()
        rs.add(maps[e0:e1], Ke)
        t_add += time.perf_counter() - t0
    t0 = time.perf_counter()
    rs.loads(m.load)
    t_add += time.perf_counter() - t0
    del Cs, maps
    rp, col, val, b = rs.export()
    csr = bo.Csr(m.ndof, rp, col, val)
    del rp, col, val
    ka, kb = args.ref_iters_a, args.ref_iters_b
    x0 = np.where(np.asarray(m.restrained, bool), m.prescribed, 0.0)
    t0 = time.perf_counter()
    rc, _, st, trace = csr.pcg(b, args.tol, maxit=200000, threads=th, rule=bo.Csr.RULE_RB, x0=x0,
                               trace_len=kb + 64)
    t_port = time.perf_counter() - t0
    if rc:
        raise RuntimeError("the oracle's solve of the reference's system did not converge")
    pa, pb = _eps_after(trace, ka), _eps_after(trace, kb)
    if pa is None or pb is None or pb[0] <= pa[0]:
        raise RuntimeError("no stop tolerances for the bounded solves")
    (ka, eps_a), (kb, eps_b) = pa, pb
    # the reference's solve at eps_b must stop after exactly kb iterations:
    # its iterate equals the oracle's kb-th (the neighbouring iterates differ
    # by far more than rounding)
    zero = np.zeros(m.ndof)
    _, xr = rs.solve(eps_b, x0=zero, want_x=True)
    _, xo, _, _ = csr.pcg(b, 0.0, maxit=kb, threads=th, rule=bo.Csr.RULE_REF, x0=x0)
    chk = float(np.linalg.norm(xr - xo) / np.linalg.norm(xo))
    if not chk <= 1e-9:
        raise RuntimeError(f"the reference's bounded solve is not the oracle's {kb}-th iterate ({chk:.2e})")
    return {"rs": rs, "iters_full": st.iterations, "t_el": t_el, "t_add": t_add, "t_struct": t_struct,
            "ka": ka, "kb": kb, "eps_a": eps_a, "eps_b": eps_b, "check": chk, "t_port_solve": t_port,
            "threads": th}


def reference_cube_step(R, ndof):
    """One bounded sample: two of the reference's Equations::solve calls on the
    full system from zero, stopped after ka and kb iterations by their
    tolerances.  Per-iteration time = the difference / (kb - ka); the solve's
    fixed cost = the ka solve minus ka iterations.  Returns (DOF/s of the
    whole workload, wall seconds of the sample, seconds per iteration)."""
    zero = np.zeros(ndof)
    ta, _ = R["rs"].solve(R["eps_a"], x0=zero)
    tb, _ = R["rs"].solve(R["eps_b"], x0=zero)
    t_it = max(1e-12, (tb - ta) / (R["kb"] - R["ka"]))
    t_fix = max(0.0, ta - R["ka"] * t_it)
    total = R["t_el"] + R["t_add"] + t_fix + R["iters_full"] * t_it
    return ndof / total, ta + tb, t_it, t_fix


def _unavailable(why):
    return {"impl": "reference", "unavailable": why}


def run_reference(args):
    """The reference's own CPU path (oracle/_ref) on the cube: assembly measured
    in full once, each step a bounded sample of its solve on the full system
    (the only extrapolation: iterations x measured full-size time per
    iteration).  Rank 0 alone works under torchrun."""
    ws, rank, local = _dist()
    if rank != 0:
        return None
    from oracle import beta_oracle as bo
    if not (bo.RefLeaf.available() and bo.RefEquations.available()):
        return _unavailable("oracle/_ref (the reference's sources compiled here) is absent")
    m = make_model(args.config, args.n)
    try:
        R = reference_cube_setup(m, args)
    except OSError as e:
        return _unavailable(f"oracle/_ref does not load on this host: {e}")
    vals, walls, its, fixes = [], [], [], []
    for k in range(args.warmup + args.steps):
        v, wall, t_it, t_fix = reference_cube_step(R, m.ndof)
        if k >= args.warmup:
            vals.append(v)
            walls.append(wall)
            its.append(t_it)
            fixes.append(t_fix)
    R["rs"].close()
    v = statistics.median(vals)
    solver = ("ParCGMatrix::solve (ParCG.cpp, 2 OpenMP threads)" if args.ref_solver == "parcg"
              else "SymmetricSparseMatrix::solve (sparse.cpp, serial)")
    cores = 2 if args.ref_solver == "parcg" else 1
    t_it = statistics.median(its)
    cb = {"value": v, "unit": UNIT, "cores": cores, "kind": "reference", "solver": solver,
          "sample": (f"the reference's own code compiled from its sources (oracle/_ref) on the whole "
                     f"{m.ndof}-dof system: element matrices (ElasticityElement3D B/addToKe, serial) "
                     f"{R['t_el']:.2f} s and Equations::addMatrix {R['t_add']:.2f} s, measured in full once; "
                     f"each step runs Equations::solve ({solver}) twice on the full system, stopped after "
                     f"{R['ka']} and {R['kb']} iterations by tolerance (checked against the oracle's iterate, "
                     f"{R['check']:.1e}): {t_it * 1e3:.1f} ms per iteration, {statistics.median(fixes) * 1e3:.1f} ms "
                     f"fixed; the full solve = fixed + {R['iters_full']} iterations x per-iteration time, the "
                     f"count from the oracle's threaded Jacobi-PCG on the reference's own matrix to "
                     f"||r||/||b|| <= {args.tol:g} (the only extrapolated quantity); structure "
                     f"{R['t_struct']:.2f} s untimed, as on the GPU"),
          "iterations_full_solve": R["iters_full"], "seconds_per_iteration": t_it,
          "seconds_assembly": R["t_el"] + R["t_add"],
          "port_all_cores": {"unit": UNIT, "cores": R["threads"], "kind": "port",
                             "seconds_full_solve": R["t_port_solve"],
                             "sample": "the oracle's threaded Jacobi-PCG, the same full solve (measured)"}}
    return {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * statistics.median(walls), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp64", "data": "synthetic (seeded generator)", "impl": "reference",
            "config": cube_config(m, args, ws), "cpu_baseline": cb,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# ---- transient diffusion (backward Euler) ------------------------------------
def heat_model(args):
    from betanoox_b200 import workloads as W
    return W.heat_slab(args.heat_nx, args.heat_nx, args.heat_nz, order=2)


def run_heat(args):
    """One bench step = one backward-Euler time step: solve C/dt + K (FP32,
    assembled in the first step's time; every step with --heat-reassemble) by
    FP32 inner PCG with FP64 refinement (the state u_s and the right-hand
    side stay on the device).  The timed region is args.heat_steps
    consecutive time steps from the initial bump."""
    import torch
    from betanoox_b200 import Solver, _abi, opts
    ws, rank, dev = _dist()
    _init_dist(dev)
    m = heat_model(args)
    u0 = m.meta["u0"]
    dt = args.dt
    stream = torch.cuda.Stream(device=dev)
    g = Solver(dev)
    g.lib.beta_gpu_set_stream(g.h, C.c_void_p(stream.cuda_stream))
    g.load_model(m)
    g.build_pattern()
    # Residual tolerance 1e-9: late in the run the field is smooth and an FP64
    # residual b - A x of it cannot resolve much below 1e-10 of the step's
    # right-hand side; the metric's bar is the solution error (<= 1e-8), which
    # is measured below against a tightly converged FP64 march.
    tol = args.heat_tol
    o_mp = opts(mode=_abi.MODE_MPIR, tol=tol, inner_tol=args.heat_inner_tol, profile=True)
    o_64 = opts(mode=_abi.MODE_FP64, stop_rule=_abi.STOP_RB, tol=tol, profile=True)

    def counters():
        a = (C.c_longlong * 3)()
        g.lib.beta_gpu_counters(g.h, a, 3)
        return list(a)

    def march(prec, o, nsteps):
        # k is linear, so C/dt + K is the same every step: assembled once, in the
        # first step's time (--heat-reassemble: every step, as the reference does)
        stats, ms = [], []
        with torch.cuda.stream(stream):
            for k in range(nsteps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                if k == 0 or args.heat_reassemble:
                    g.assemble(prec, _abi.ASM_MBAR, dt, 1.0)
                st, _ = g.heat_run(dt, 1, o)
                e1.record(stream)
                stats.append(st)
                ms.append((e0, e1))
        _barrier()
        return [a.elapsed_time(b) for a, b in ms], stats

    g.heat_set_state(u0)
    march(_abi.FP32, o_mp, args.warmup)
    g.heat_set_state(u0)
    _barrier()
    c0 = counters()
    with Clocks(dev) as clk:
        ms_mp, st_mp = march(_abi.FP32, o_mp, args.heat_steps)
    c1 = counters()
    u_mp = g.heat_get_state()
    tot_ms = _max_over_ranks(sum(ms_mp), dev)
    value = ws * m.ndof * args.heat_steps / (tot_ms / 1e3)
    out = None
    if rank == 0:
        fp64 = None
        if not args.skip_fp64:
            g.heat_set_state(u0)
            ms_64, st_64 = march(_abi.FP64, o_64, args.heat_steps)
            u_64 = g.heat_get_state()
            fp64 = {"value": ws * m.ndof * args.heat_steps / (sum(ms_64) / 1e3), "ms_total": sum(ms_64),
                    "iterations_per_step_median": int(statistics.median([s.iterations for s in st_64]))}
        err = None
        if not args.skip_accuracy:
            g.heat_set_state(u0)
            march(_abi.FP64, opts(mode=_abi.MODE_FP64, stop_rule=_abi.STOP_RB, tol=1e-13), args.heat_steps)
            u_t = g.heat_get_state()
            err = {"mixed": float(np.linalg.norm(u_mp - u_t) / np.linalg.norm(u_t))}
            if fp64:
                err["fp64"] = float(np.linalg.norm(u_64 - u_t) / np.linalg.norm(u_t))
        e2e = None
        if not args.skip_e2e:
            pm = type(m)(m.name, m.kind, m.ndim, _pinned_copy(m.xyz), _pinned_copy(m.conn), m.ndpn,
                         _pinned_copy(m.params), _pinned_copy(m.restrained), _pinned_copy(m.prescribed),
                         _pinned_copy(m.load), m.order, m.meta)
            u0p = _pinned_copy(u0)
            u_host = _pinned_copy(np.zeros(m.ndof))
            ge = Solver(dev)
            ge.lib.beta_gpu_set_stream(ge.h, C.c_void_p(stream.cuda_stream))
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            ge.load_model(pm)
            ge.build_pattern()
            ge.lib.beta_gpu_heat_set_state(ge.h, u0p.ctypes.data_as(C.c_void_p))
            for k in range(args.heat_steps):
                if k == 0 or args.heat_reassemble:
                    ge.assemble(_abi.FP32, _abi.ASM_MBAR, dt, 1.0)
                ge.heat_run(dt, 1, o_mp)
            ge.lib.beta_gpu_heat_get_state(ge.h, u_host.ctypes.data_as(C.c_void_p))
            torch.cuda.synchronize()
            tw = time.perf_counter() - t1
            a = (C.c_longlong * 3)()
            ge.lib.beta_gpu_counters(ge.h, a, 3)
            e2e = {"value": ws * m.ndof * args.heat_steps / tw, "unit": UNIT, "h2d_bytes_per_step": a[1],
                   "d2h_bytes_per_step": a[2], "ms_per_step": 1e3 * tw,
                   "includes": f"upload, host structure, {args.heat_steps} x (FP32 assembly + solve), download; "
                               f"a step here is the whole {args.heat_steps}-step run"}
            ge.close()
        peak, peak_kind = _peaks()
        spmv_ms = statistics.median([s.ms_spmv_avg for s in st_mp])
        layout = g.block_layout()
        alg = spmv_algorithmic_bytes(_nblk(m), m.nnode, 1, layout[2])
        achieved = alg / (spmv_ms * 1e-3) / 1e9 if spmv_ms > 0 else None
        tr = _traffic("spmv_traffic_heat.json")
        kern = _layout_label(layout, 1)
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None,
                "traffic": (round(tr["traffic_over_algorithmic"] * alg)
                            if tr and tr.get("kernel") == kern.split(" ")[0] else None),
                "kernel": kern + ", one dof per node",
                "algorithmic_bytes_per_launch": alg, "ms_per_launch": spmv_ms,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                else "fallback 6.65 TB/s"}
        its = [s.iterations for s in st_mp]
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.heat_steps,
            "warmup": args.warmup, "ms_per_step": tot_ms / args.heat_steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp32 inner / fp64 outer",
            "data": "synthetic (seeded generator)",
            "config": {"workload": f"transient diffusion hex8 {args.heat_nx}x{args.heat_nx}x{args.heat_nz}, "
                                   f"{m.ndof} dofs, backward Euler dt={dt}, k=exp(N(0,1)), c=1, T=0 on all faces, "
                                   f"Gaussian bump, 2x2x2 Gauss; "
                                   + ("each step assembles C/dt+K (FP32) and solves it" if args.heat_reassemble
                                      else "C/dt+K (FP32) assembled once in the first step (k linear), "
                                           "each step solves it"),
                       "ndof": m.ndof, "time_steps": args.heat_steps, "tol": tol,
                       "parallelism": f"replicas x{ws}", "l2": "inputs larger than L2 (matrix ~1 GB)"},
            "per_step_ms": {"p50": float(np.percentile(ms_mp, 50)), "p99": float(np.percentile(ms_mp, 99))},
            "heat": {"iterations_per_step": [min(its), int(statistics.median(its)), max(its)],
                     "refinements_per_step_median": int(statistics.median([s.outer_iterations for s in st_mp]))},
            "e2e": e2e, "gpu_launches": c1[0] - c0[0], "roofline": roof, "clocks": clk.summary(),
        }
        if fp64:
            out["fp64_plain"] = fp64
            out["mixed_over_fp64"] = value / fp64["value"]
        if err:
            out["rel_err_vs_fp64_reference"] = err
        if not args.skip_cpu:
            out["cpu_baseline"] = heat_cpu_baseline(args, m)
    g.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return out


def heat_cpu_baseline(args, m):
    """The reference transient step on the host (oracle restatement: FP64
    assembly of Mbar and F, threaded Jacobi-PCG) on a smaller slab with the
    same cell size ratio, a few steps, scaled to the full workload by dofs."""
    from oracle import beta_oracle as bo
    from betanoox_b200 import workloads as W
    nx, nz = args.cpu_heat_nx, max(2, args.cpu_heat_nx * args.heat_nz // args.heat_nx)
    ms = W.heat_slab(nx, nx, nz, order=2)
    s = bo.System(ms)
    s.set_bc(ms.restrained, ms.prescribed, ms.load)
    s.build_pattern()
    u = ms.meta["u0"].copy()
    t0 = time.perf_counter()
    k = 0
    while k < 2 or (time.perf_counter() - t0 < 10.0 and k < 20):
        s.set_bc(ms.restrained, ms.prescribed, ms.load)
        rc, u, st = s.heat_step(ms.params, ms.order, args.dt, u, eps=args.heat_tol, maxit=100000)
        k += 1
    per_dof_step = (time.perf_counter() - t0) / k / ms.ndof
    return {"value": 1.0 / per_dof_step, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{k} backward-Euler steps of the {nx}x{nx}x{nz} slab ({ms.ndof} dofs) on one host thread "
                      f"(FP64 assembly + Jacobi-PCG), rate per dof applied to the {m.ndof}-dof workload"}


def reference_heat_baseline(args, m):
    """The transient step by the reference's own code (oracle/_ref) on the
    port's sample slab: per element K and M through its addToKe / addToMe,
    formK_s / formF_s_new, then Equations::addMatrix and the solve from u_s
    (the structure is built once per analysis, as the reference does, and not
    timed).  Each step's state is first advanced by the oracle's step, which
    proves convergence (the reference's solve exits otherwise) and is timed as
    the one-thread port on the same steps.  None when oracle/_ref is absent."""
    from oracle import beta_oracle as bo
    from betanoox_b200 import workloads as W
    if not (bo.RefLeaf.available() and bo.RefEquations.available()):
        return None
    leaf, req = bo.RefLeaf(), bo.RefEquations()
    nx, nz = args.cpu_heat_nx, max(2, args.cpu_heat_nx * args.heat_nz // args.heat_nx)
    ms = W.heat_slab(nx, nx, nz, order=m.order)
    maps = (ms.first_dof[ms.conn][:, :, None] + np.arange(ms.ndpn)[None, None, :]).reshape(ms.nelem, ms.nnpe)
    xe = np.ascontiguousarray(ms.xyz[ms.conn])
    s = bo.System(ms)
    s.set_bc(ms.restrained, ms.prescribed, ms.load)
    s.build_pattern()
    u = ms.meta["u0"].copy()
    t_ref = t_port = 0.0
    k = 0
    while k < 2 or (t_ref + t_port < 10.0 and k < 20):
        t0 = time.perf_counter()
        s.set_bc(ms.restrained, ms.prescribed, ms.load)
        rc, u_next, st = s.heat_step(ms.params, ms.order, args.dt, u, eps=args.heat_tol, maxit=100000)
        t_port += time.perf_counter() - t0
        if rc != 0:
            return None
        ue = u[maps]
        t0 = time.perf_counter()
        Mb, F = leaf.heat_hex8_step_terms(xe, ms.params[:, :3], ms.params[:, 3], ms.order, ue, args.dt, 0.0, args.dt)
        t_el = time.perf_counter() - t0
        secs = []
        req.assemble(ms.ndof, maps, Mb, ms.restrained, ms.prescribed, ms.load, solve=True, eps=args.heat_tol,
                     maxit=100000, Fe=F, x0=u, timings=secs)
        t_ref += t_el + secs[1] + secs[2]
        u = u_next
        k += 1
    return {"value": ms.ndof * k / t_ref, "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": (f"{k} backward-Euler steps of the {nx}x{nx}x{nz} slab ({ms.ndof} dofs) by the reference's "
                       f"own code compiled from its sources (oracle/_ref): element K/M (addToKe/addToMe), "
                       f"formK_s/formF_s_new, Equations::addMatrix and SymmetricSparseMatrix::solve, one host "
                       f"thread; rate per dof applied to the {m.ndof}-dof workload"),
            "port_single_thread": {"value": ms.ndof * k / t_port, "unit": UNIT, "cores": 1, "kind": "port",
                                   "sample": f"the oracle's step on the same {k} steps"}}


def run_heat_reference(args):
    """The reference's own transient step (oracle/_ref) on a bounded sample
    slab; each bench step is one such sample.  Prints the unavailable line
    where oracle/_ref is absent or does not load."""
    ws, rank, _ = _dist()
    if rank != 0:
        return None
    from oracle import beta_oracle as bo
    if not (bo.RefLeaf.available() and bo.RefEquations.available()):
        return _unavailable("oracle/_ref (the reference's sources compiled here) is absent")
    m = heat_model(args)
    vals, walls, cb = [], [], None
    try:
        for k in range(args.warmup + max(1, args.steps)):
            t0 = time.perf_counter()
            cb = reference_heat_baseline(args, m)
            wall = time.perf_counter() - t0
            if cb is None:
                return _unavailable("the oracle's transient step did not converge on the sample slab")
            if k >= args.warmup:
                vals.append(cb["value"])
                walls.append(wall)
    except OSError as e:
        return _unavailable(f"oracle/_ref does not load on this host: {e}")
    v = statistics.median(vals)
    cb["value"] = v
    return {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * statistics.median(walls), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp64", "data": "synthetic (seeded generator)", "impl": "reference",
            "config": {"workload": f"transient diffusion hex8 {args.heat_nx}x{args.heat_nx}x{args.heat_nz}, "
                                   f"{m.ndof} dofs, backward Euler dt={args.dt}", "ndof": m.ndof},
            "cpu_baseline": cb, "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# ---- batched RVEs (one persistent launch) ---------------------------------
def iter_bytes(nblk, nnode, nd):
    """Algorithmic bytes of one inner FP32 PCG iteration of the batched solver
    for one system: SpMV (every stored block's nd*nd values + column index, the
    direction gathered once, q written once), the update pass (y, r, q, p and
    the packed block-Jacobi factor read; y, r written) and the direction pass
    (r, p, factor read; p written).  p is padded to float4 for nd = 3."""
    nd4 = 4 * nd
    pv = 16 if nd == 3 else nd4
    mv = 4 * nd * (nd + 1) // 2
    return nblk * (4 * nd * nd + 4) + nnode * (7 * nd4 + 4 * pv + 2 * mv)


def structured_nblk(m):
    """Node-pair blocks of a structured n^3 hex8 cube: the node graph is the
    tensor product of three 1-D graphs with 3n+1 entries each."""
    n = int(m.meta["n"])
    return (3 * n + 1) ** 3


def cpu_full_solves(models, tol, budget_s, threads):
    """The reference algorithm on the host (oracle restatement): structure,
    FP64 assembly and threaded Jacobi-PCG (stop rule sqrt(r.r/x.x) < tol) of
    whole systems, in list order, until budget_s seconds have been spent."""
    from oracle import beta_oracle as bo
    done, dofs, secs = 0, 0, 0.0
    for m in models:
        t0 = time.perf_counter()
        s = bo.System(m)
        s.set_bc(m.restrained, m.prescribed, m.load)
        s.build_pattern()
        s.assemble(m.params, m.order)
        rc, x, st = s.solve_threaded(s.rhs(), tol, maxit=200000, threads=threads)
        secs += time.perf_counter() - t0
        done += 1
        dofs += m.ndof
        del s
        if secs >= budget_s:
            break
    return done, dofs, secs


def reference_full_solves(models, tol, budget_s, threads):
    """Whole systems, in list order until budget_s seconds are spent, solved by
    the reference's own code (oracle/_ref): element matrices through its
    elements (ElasticityElement3D / ElasticityElement2D B and addToKe, or
    HeatTransferElement3Dtransient addToKe for steady diffusion), the
    Equations pattern, addMatrix and its two-thread ParCG solve (stop rule
    sqrt(r.r/x.x) < tol).  Each system
    is first solved by the oracle's threaded port, which proves convergence
    (the reference's solve exits otherwise) and gives the port's time on the
    same systems.  Returns (systems, dofs, reference seconds, port seconds), or
    None when oracle/_ref is absent."""
    from oracle import beta_oracle as bo
    if not (bo.RefLeaf.available() and bo.RefEquations.available()):
        return None
    leaf, req = bo.RefLeaf(), bo.RefEquations()
    done, dofs, t_ref, t_port = 0, 0, 0.0, 0.0
    for m in models:
        t0 = time.perf_counter()
        s = bo.System(m)
        s.set_bc(m.restrained, m.prescribed, m.load)
        s.build_pattern()
        s.assemble(m.params, m.order)
        rc, _, _ = s.solve_threaded(s.rhs(), tol, maxit=200000, threads=threads)
        t_port += time.perf_counter() - t0
        del s
        if rc != 0:
            break
        # one material matrix per distinct parameter row (the reference's
        # material objects are per group), built before the clock starts
        rows, inv = np.unique(m.params, axis=0, return_inverse=True)
        inv = np.asarray(inv).reshape(-1)
        nd = m.nnpe * m.ndpn
        maps = (m.first_dof[m.conn][:, :, None] + np.arange(m.ndpn)[None, None, :]).reshape(m.nelem, nd)
        xe = np.ascontiguousarray(m.xyz[m.conn])
        if m.kind == 2:    # hex8 elasticity
            C = np.stack([bo.cmat_ortho3d(r) for r in rows])[inv]
            element = lambda: leaf.elastic_hex8_ke(xe, C, m.order)  # noqa: E731
        elif m.kind == 1:  # quad4 plane stress
            C = np.stack([bo.cmat_plane_stress(r[:4]) for r in rows])[inv]
            element = lambda: leaf.elastic_quad4_ke(xe, C, m.order)  # noqa: E731
        elif m.kind == 3:  # hex8 diffusion, steady
            k3 = np.ascontiguousarray(m.params[:, :3])
            element = lambda: leaf.heat_hex8_k(xe, k3, m.order)  # noqa: E731
        else:
            break
        t0 = time.perf_counter()
        Ke = element()
        req.assemble(m.ndof, maps, Ke, m.restrained, m.prescribed, m.load, solve=True, eps=tol, maxit=200000,
                     parcg=True)
        t_ref += time.perf_counter() - t0
        done += 1
        dofs += m.ndof
        if t_ref + t_port >= budget_s:
            break
    return done, dofs, t_ref, t_port


def run_batch(args, nested=False):
    """The batch configuration.  nested: a sub-record of the default line (the
    process group already exists and stays up; no CPU baseline)."""
    import torch
    from betanoox_b200 import Batch, Solver, _abi, opts
    from betanoox_b200 import workloads as W
    ws, rank, dev = _dist()
    if not nested:
        _init_dist(dev)
    t0 = time.perf_counter()
    models = W.rve_batch(count=args.count, seed=args.seed)
    t_gen = time.perf_counter() - t0
    ndof_tot = sum(m.ndof for m in models)
    o = opts(mode=_abi.MODE_MPIR, tol=args.tol, inner_tol=args.inner_tol)
    b = Batch(dev, hbm_budget=int(args.pool_gb * (1 << 30)), max_systems=len(models) + 8)
    t0 = time.perf_counter()
    ids = b.add_many(models)
    t_add = time.perf_counter() - t0
    assert all(i is not None for i in ids), "pool too small for the batch"
    t0 = time.perf_counter()
    if args.shape:
        threads, boost = (int(v) for v in args.shape.split(","))
        b.tune(threads, boost)
    else:
        threads, boost = b.autotune(o, budget=args.tune_iters)
    t_tune = time.perf_counter() - t0
    for _ in range(args.warmup):
        b.reset()
        b.run(o)
    _barrier()
    ms = []
    l0 = b.info()["launches"]
    with Clocks(dev) as clk:
        for _ in range(args.steps):
            b.reset()
            left = b.run(o)
            assert left == 0
            ms.append(b.info()["last_launch_ns"] / 1e6)
    launches = b.info()["launches"] - l0
    ginfo = b.info()
    _barrier()
    res = [b.result(i, with_u=False) for i in ids]
    bad = [(models[k].name, _abi.STATUS_NAMES.get(r[0])) for k, r in enumerate(res) if r[0] != _abi.OK]
    iters = [r[2].iterations for r in res]
    tot_ms = _max_over_ranks(sum(ms), dev)
    value = ws * ndof_tot * args.steps / (tot_ms / 1e3)

    out = None
    if rank == 0:
        # accuracy on a sample: batch solution vs a tight plain FP64 GPU solve
        errs = []
        fp64_ms, fp64_dofs, fp64_iters = 0.0, 0, []
        stream = torch.cuda.Stream(device=dev)
        for k, (sid, m) in enumerate(zip(ids, models)):
            want_acc = k % args.check_every == 0
            want_64 = k % args.fp64_stride == 0 and k // args.fp64_stride < args.fp64_sample
            if not (want_acc or want_64):
                continue
            g = Solver(dev)
            g.lib.beta_gpu_set_stream(g.h, C.c_void_p(stream.cuda_stream))
            g.load_model(m)
            g.build_pattern()
            if want_64:
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                with torch.cuda.stream(stream):
                    e0.record(stream)
                    g.assemble(_abi.FP64)
                    rc, st = g.solve(opts(mode=_abi.MODE_FP64, stop_rule=_abi.STOP_RB, tol=args.tol))
                    e1.record(stream)
                stream.synchronize()
                fp64_ms += e0.elapsed_time(e1)
                fp64_dofs += m.ndof
                fp64_iters.append(st.iterations)
            if want_acc:
                g.assemble(_abi.FP64)
                g.solve(opts(mode=_abi.MODE_FP64, stop_rule=_abi.STOP_RB, tol=1e-13))
                ut = g.download()
                _, u, _ = b.result(sid)
                errs.append(float(np.linalg.norm(u - ut) / np.linalg.norm(ut)))
            g.close()
        # end to end: host models in, solutions out, through the batch API
        e2e = None
        if not args.skip_e2e:
            tw = []
            for _ in range(max(1, args.e2e_steps)):
                t1 = time.perf_counter()
                be = Batch(dev, hbm_budget=int(args.pool_gb * (1 << 30)), max_systems=len(models) + 8)
                be.tune(threads, boost)
                eids = be.add_many(models)
                be.run(o)
                for sid in eids:
                    be.result(sid)
                tw.append(time.perf_counter() - t1)
                inf = be.info()
                be.close()
            e2e = {"value": ws * ndof_tot / statistics.median(tw), "unit": UNIT,
                   "h2d_bytes_per_step": inf["h2d"], "d2h_bytes_per_step": inf["d2h"],
                   "ms_per_step": 1e3 * statistics.median(tw),
                   "includes": "host structure build (all cores), pool upload, one launch, solution download"}
        peak, peak_kind = _peaks()
        ms_launch = statistics.median(ms)
        alg = sum(it * iter_bytes(structured_nblk(m), m.nnode, 3) for it, m in zip(iters, models))
        achieved = alg / (ms_launch * 1e-3) / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": None, "kernel": f"k_batch_solve<{threads}> (gang boost {boost}): assembly + all PCG",
                "algorithmic_bytes_per_launch": alg, "ms_per_launch": ms_launch,
                "note": "inner-iteration bytes only (assembly and FP64 residual replacements excluded); "
                        "small systems re-read their matrix from L2",
                "ncu_dram": _traffic("batch_dram.json"),
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                else "fallback 6.65 TB/s"}
        sizes = sorted(m.meta["n"] for m in models)
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tot_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp32 inner / fp64 outer",
            "data": "synthetic (seeded generator)",
            "config": {"workload": f"{len(models)} two-phase RVE hex8 cubes n~U{{8..40}} "
                                   f"(n {sizes[0]}..{sizes[-1]}), {ndof_tot} dofs total, one persistent launch",
                       "global_batch": ws * len(models), "ndof_total": ndof_tot, "parallelism": f"replicas x{ws}",
                       "tol": args.tol, "stop_rule": "||b-Au||/||b||",
                       "launch_shape": {"threads": threads, "gang_boost": boost, "gangs": ginfo["gangs"],
                                        "gang_ctas": ginfo["gang_ctas"]},
                       "l2": f"inputs larger than L2 (pool {b.info()['used'] / 2**30:.1f} GiB)"},
            "per_step_ms": {"p50": float(np.percentile(ms, 50)), "p99": float(np.percentile(ms, 99))},
            "batch": {"ms_steps": ms, "iterations_total": int(sum(iters)), "iterations_max": int(max(iters)),
                      "not_converged": bad[:5], "n_not_converged": len(bad), "setup_s": {"generate": t_gen,
                      "add_many": t_add, "autotune": t_tune},
                      "group_time_share": _phase_shares(b.info()),
                      # the systems whose groups ran longest in the last launch, against the launch
                      "longest_systems": [{"n": models[k].meta["n"], "iterations": res[k][2].iterations,
                                           "group_ms": round(res[k][2].ms_solve, 2)}
                                          for k in sorted(range(len(res)), key=lambda k: -res[k][2].ms_solve)[:4]]},
            "e2e": e2e, "gpu_launches": launches, "roofline": roof, "clocks": clk.summary(),
        }
        if errs:
            out["rel_err_vs_fp64_reference"] = {"max": max(errs), "n_checked": len(errs)}
        if fp64_dofs:
            v64 = fp64_dofs / (fp64_ms / 1e3)
            out["fp64_plain"] = {"value": ws * v64, "systems": len(fp64_iters),
                                 "how": f"sequential per-system plain FP64 Jacobi-PCG (FP64 assembly + solve, "
                                        f"CUDA events), same stop rule and tol, on every {args.fp64_stride}-th "
                                        f"system of the batch",
                                 "iterations_median": int(statistics.median(fp64_iters))}
            out["mixed_over_fp64"] = value / (ws * v64)
        if not args.skip_cpu and not nested:
            th = os.cpu_count() or 1
            n, d, sec = cpu_full_solves(models, args.tol, args.cpu_budget_s, th)
            out["cpu_baseline"] = {"value": d / sec, "unit": UNIT, "cores": th, "kind": "port",
                                   "sample": f"first {n} of {len(models)} RVEs solved whole on the host "
                                             f"({d} dofs in {sec:.1f} s): FP64 assembly + threaded Jacobi-PCG"}
    b.close()
    if ws > 1 and not nested:
        import torch.distributed as dist
        dist.destroy_process_group()
    return out


def run_batch_reference(args):
    """Whole RVEs of the batch, in list order within a time budget per step,
    solved by the reference's own code (oracle/_ref) one system at a time;
    each bench step is one such sample.  Prints the unavailable line where
    oracle/_ref is absent or does not load."""
    ws, rank, _ = _dist()
    if rank != 0:
        return None
    from oracle import beta_oracle as bo
    if not (bo.RefLeaf.available() and bo.RefEquations.available()):
        return _unavailable("oracle/_ref (the reference's sources compiled here) is absent")
    from betanoox_b200 import workloads as W
    models = W.rve_batch(count=args.count, seed=args.seed)
    ndof_tot = sum(m.ndof for m in models)
    th = os.cpu_count() or 1
    rvals, pvals, walls, ref = [], [], [], None
    try:
        for k in range(args.warmup + max(1, args.steps)):
            t0 = time.perf_counter()
            ref = reference_full_solves(models, args.tol, args.cpu_budget_s / max(1, args.steps), th)
            wall = time.perf_counter() - t0
            if ref is None or ref[0] == 0:
                return _unavailable("no RVE was solved by the reference's code within the step's budget")
            if k >= args.warmup:
                rvals.append(ref[1] / ref[2])
                pvals.append(ref[1] / ref[3])
                walls.append(wall)
    except OSError as e:
        return _unavailable(f"oracle/_ref does not load on this host: {e}")
    n, d, t_ref, t_port = ref
    v = statistics.median(rvals)
    return {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * statistics.median(walls), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp64", "data": "synthetic (seeded generator)",
            "impl": "reference",
            "config": {"workload": f"{len(models)} two-phase RVE hex8 cubes n~U{{8..40}}, {ndof_tot} dofs total",
                       "ndof_total": ndof_tot},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": 2, "kind": "reference",
                             "sample": f"first {n} RVEs solved whole per step ({d} dofs, {t_ref:.1f} s) by the "
                                       f"reference's own code compiled from its sources (oracle/_ref): "
                                       f"element B/addToKe, Equations pattern + addMatrix, ParCG solve, "
                                       f"one system at a time; the rate applies to the whole batch",
                             "port_all_cores": {"value": statistics.median(pvals), "unit": UNIT, "cores": th,
                                                "kind": "port",
                                                "sample": f"the same {n} RVEs, FP64 assembly + threaded "
                                                          f"Jacobi-PCG ({t_port:.1f} s)"}},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# ---- serving: Poisson stream through the continuous-batching server ---------
def _serve_stream(server, models, arrivals, threads):
    """Submits models[j % len(models)] at arrivals[j] seconds (from a pool of
    submitter threads, which build each request's structure), collects every
    result, and returns per-request (latency s, dofs, state, status, final_norm)
    and the wall time from the first arrival to the last completion."""
    import queue
    from betanoox_b200 import _abi
    n = len(arrivals)
    q = queue.Queue()
    subs = [None] * n  # (rid, t_submit_start, t_submit_end)
    t_base = time.perf_counter() + 0.05

    def submitter():
        while True:
            j = q.get()
            if j is None:
                return
            m = models[j % len(models)]
            ts = time.perf_counter()
            rid = server.submit(m)
            subs[j] = (rid, ts)

    pool = [threading.Thread(target=submitter, daemon=True) for _ in range(threads)]
    for t in pool:
        t.start()
    for j in range(n):
        now = time.perf_counter() - t_base
        if arrivals[j] > now:
            time.sleep(arrivals[j] - now)
        q.put(j)
    for _ in pool:
        q.put(None)
    for t in pool:
        t.join()
    out = []
    t_end = 0.0
    for j in range(n):
        rid, ts = subs[j]
        state, _, st, lat_ms = server.wait(rid, timeout_s=600.0)
        done_at = (ts - t_base) + lat_ms / 1e3
        t_end = max(t_end, done_at)
        out.append(((done_at - arrivals[j]), models[j % len(models)].ndof, state, st.status, st.final_norm))
    return out, t_end - arrivals[0]


def run_serve(args, nested=False):
    """The serving configuration.  nested: a sub-record of the default line
    (the process group already exists and stays up; no CPU baseline)."""
    import torch
    from betanoox_b200 import Server, _abi, opts
    from betanoox_b200 import workloads as W
    ws, rank, dev = _dist()
    if not nested:
        _init_dist(dev)
    t0 = time.perf_counter()
    pool_n = min(args.requests, args.serve_pool)
    models = [W.serve_request(args.seed + 1000 * rank, j) for j in range(pool_n)]
    t_gen = time.perf_counter() - t0
    o = opts(mode=_abi.MODE_MPIR, tol=args.tol, inner_tol=args.inner_tol)
    th = args.submit_threads or (os.cpu_count() or 1)
    srv = Server(dev, hbm_budget=int(args.pool_gb * (1 << 30)), max_systems=4096, o=o,
                 iters_per_launch=args.iters_per_launch, threads=args.threads, gang_boost=args.gang_boost,
                 slice_us=args.slice_us)
    # capacity: a burst of the first `cap` pool models submitted at once
    cap_n = min(args.capacity_requests, pool_n)
    for _ in range(args.warmup):
        _serve_stream(srv, models[:min(cap_n, 32)], np.zeros(min(cap_n, 32)), th)
    sc0 = srv.stats()
    with Clocks(dev) as clk_cap:
        res_cap, wall_cap = _serve_stream(srv, models[:cap_n], np.zeros(cap_n), th)
    sc1 = srv.stats()
    cap_busy = (sc1["busy_us"] - sc0["busy_us"]) / 1e6 / wall_cap
    cap_rps = cap_n / wall_cap
    cap_dofs = sum(r[1] for r in res_cap) / wall_cap
    lam = args.load * cap_rps
    rng = np.random.default_rng(args.seed)
    arrivals = np.cumsum(rng.exponential(1.0 / lam, size=args.requests))
    arrivals -= arrivals[0]
    s0 = srv.stats()
    _barrier()
    with Clocks(dev) as clk:
        res, wall = _serve_stream(srv, models, arrivals, th)
    s1 = srv.stats()
    wall = _max_over_ranks(wall, dev)
    lat = np.array([r[0] for r in res]) * 1e3
    dofs = sum(r[1] for r in res)
    states = [r[2] for r in res]
    value = ws * dofs / wall
    out = None
    if rank == 0:
        ok = sum(1 for r in res if r[2] == _abi.REQ_DONE and r[3] == _abi.OK)
        # plain FP64 GPU PCG, one request at a time end to end (same API level)
        fp64 = None
        if args.serve_fp64_sample:
            from betanoox_b200 import Solver
            tw, d64 = 0.0, 0
            # one context for every request, as a single-system server would
            # keep it (its buffers are reused; a context per request would add
            # its creation and teardown to each request)
            g = Solver(dev)
            ph = np.zeros(5)
            o64 = opts(mode=_abi.MODE_FP64, stop_rule=_abi.STOP_RB, tol=args.tol)
            # a sample spread evenly over the pool, so that its sizes and
            # families follow the stream's
            stride = max(1, len(models) // max(1, args.serve_fp64_sample))
            sample = models[::stride][:args.serve_fp64_sample]
            for m in sample:
                t = [time.perf_counter()]
                g.load_model(m)
                t.append(time.perf_counter())
                g.build_pattern()
                t.append(time.perf_counter())
                g.assemble(_abi.FP64)
                t.append(time.perf_counter())
                g.solve(o64)
                t.append(time.perf_counter())
                g.download()
                t.append(time.perf_counter())
                ph += np.diff(t)
                tw += t[-1] - t[0]
                d64 += m.ndof
            g.close()
            fp64 = {"value": ws * d64 / tw, "requests": len(sample), "sample": f"every {stride}-th request",
                    "phases_s": dict(zip(["upload", "structure", "assembly", "solve", "download"],
                                         [round(float(v), 4) for v in ph])),
                    "how": "sequential requests through the single-system API on one reused context, plain "
                           "FP64 Jacobi-PCG: host structure build + upload + assembly + solve + download"}
        fams = {}
        for j in range(len(res)):
            f = models[j % len(models)].meta["family"]
            fams[f] = fams.get(f, 0) + 1
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": 1, "warmup": args.warmup,
            "ms_per_step": wall * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "fp32 inner / fp64 outer", "data": "synthetic (seeded generator)",
            "config": {"workload": f"Poisson stream of {args.requests} requests (quad4 / hex8 elasticity / hex8 "
                                   f"diffusion, log-uniform 1e3-5e5 dofs) at {args.load:.0%} of measured capacity",
                       "requests": args.requests, "distinct_models": pool_n, "families": fams,
                       "lambda_per_s": lam, "capacity_req_per_s": cap_rps, "tol": args.tol,
                       "iters_per_launch": args.iters_per_launch, "slice_us": args.slice_us, "submit_threads": th,
                       "launch_shape": {"threads": args.threads, "gang_boost": args.gang_boost},
                       "parallelism": f"replicas x{ws}",
                       "l2": "working set above L2 (pool of resident systems)"},
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "mean": float(lat.mean()), "max": float(lat.max())},
            "serve": {"done_ok": ok, "states": {str(k): states.count(k) for k in set(states)},
                      "max_final_norm": float(max(r[4] for r in res)), "launches": s1["launches"] - s0["launches"],
                      "busy_frac": (s1["busy_us"] - s0["busy_us"]) / 1e6 / wall, "wall_s": wall,
                      "generate_s": t_gen,
                      "capacity_burst": {"requests": cap_n, "wall_s": wall_cap, "dofs_per_s": cap_dofs,
                                         "busy_frac": cap_busy, "group_time_share": _phase_shares(sc1, sc0),
                                         "clocks": clk_cap.summary()},
                      "group_time_share": _phase_shares(s1, s0)},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": s1["h2d"] - s0["h2d"],
                    "d2h_bytes_per_step": s1["d2h"] - s0["d2h"],
                    "includes": "arrival to result on host: structure build, admission, solve, download"},
            "gpu_launches": s1["launches"] - s0["launches"], "clocks": clk.summary(),
        }
        if fp64:
            out["fp64_plain"] = fp64
            out["mixed_over_fp64"] = value / fp64["value"]
            out["capacity_over_fp64"] = cap_dofs / fp64["value"]
        if not args.skip_cpu and not nested:
            thc = os.cpu_count() or 1
            n, d, sec = cpu_full_solves(models, args.tol, args.cpu_budget_s, thc)
            out["cpu_baseline"] = {"value": d / sec, "unit": UNIT, "cores": thc, "kind": "port",
                                   "sample": f"first {n} requests solved whole on the host, one at a time "
                                             f"({d} dofs in {sec:.1f} s): FP64 assembly + threaded Jacobi-PCG"}
    srv.close()
    if ws > 1 and not nested:
        import torch.distributed as dist
        dist.destroy_process_group()
    return out


def run_serve_reference(args):
    """The request stream's first requests solved whole, one at a time, by the
    reference's own code (oracle/_ref) within a time budget per step; each
    bench step is one such sample.  Prints the unavailable line where
    oracle/_ref is absent or does not load."""
    ws, rank, _ = _dist()
    if rank != 0:
        return None
    from oracle import beta_oracle as bo
    if not (bo.RefLeaf.available() and bo.RefEquations.available()):
        return _unavailable("oracle/_ref (the reference's sources compiled here) is absent")
    from betanoox_b200 import workloads as W
    pool_n = min(args.requests, args.serve_pool)
    models = [W.serve_request(args.seed, j) for j in range(pool_n)]
    th = os.cpu_count() or 1
    rvals, pvals, walls, ref = [], [], [], None
    try:
        for k in range(args.warmup + max(1, args.steps)):
            t0 = time.perf_counter()
            ref = reference_full_solves(models, args.tol, args.cpu_budget_s / max(1, args.steps), th)
            wall = time.perf_counter() - t0
            if ref is None or ref[0] == 0:
                return _unavailable("no request was solved by the reference's code within the step's budget")
            if k >= args.warmup:
                rvals.append(ref[1] / ref[2])
                pvals.append(ref[1] / ref[3])
                walls.append(wall)
    except OSError as e:
        return _unavailable(f"oracle/_ref does not load on this host: {e}")
    n, d, t_ref, t_port = ref
    v = statistics.median(rvals)
    return {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * statistics.median(walls), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp64", "data": "synthetic (seeded generator)",
            "impl": "reference",
            "config": {"workload": f"stream of {args.requests} requests (quad4 / hex8 elasticity / hex8 "
                                   f"diffusion, log-uniform 1e3-5e5 dofs), solved one at a time"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": 2, "kind": "reference",
                             "sample": f"first {n} requests solved whole per step ({d} dofs, {t_ref:.1f} s) by "
                                       f"the reference's own code compiled from its sources (oracle/_ref): "
                                       f"its elements, Equations pattern + addMatrix, ParCG solve",
                             "port_all_cores": {"value": statistics.median(pvals), "unit": UNIT, "cores": th,
                                                "kind": "port", "sample": f"the same {n} requests ({t_port:.1f} s)"}},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="cube")
    ap.add_argument("--n", type=int, default=100)
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--inner-tol", type=float, default=0.01)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--skip-fp64", action="store_true")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-accuracy", action="store_true")
    # the oracle's accuracy reference: ||r||/||b|| of its FP64 solution
    ap.add_argument("--oracle-tol", type=float, default=1e-12)
    # the reference arm's bounded solves: iteration counts of the two samples
    # per step, and the reference's solver (ParCG: its two-thread OpenMP one)
    ap.add_argument("--ref-iters-a", type=int, default=2)
    ap.add_argument("--ref-iters-b", type=int, default=6)
    ap.add_argument("--ref-solver", default="parcg", choices=["parcg", "serial"])
    ap.add_argument("--cpu-budget-s", type=float, default=20.0)
    # batch / serve
    ap.add_argument("--count", type=int, default=512)
    ap.add_argument("--seed", type=int, default=99)
    ap.add_argument("--pool-gb", type=float, default=48.0)
    ap.add_argument("--tune-iters", type=int, default=0, help="0: autotune on complete solves")
    ap.add_argument("--check-every", type=int, default=32)
    ap.add_argument("--shape", default="", help="threads,gang_boost: skip the autotuner")
    ap.add_argument("--fp64-sample", type=int, default=512)
    ap.add_argument("--fp64-stride", type=int, default=1, help="batch: plain FP64 on every k-th system")
    # the batched and served forms inside the default (cube) line
    ap.add_argument("--skip-batch", action="store_true")
    ap.add_argument("--skip-serve", action="store_true")
    ap.add_argument("--sub-steps", type=int, default=3)
    ap.add_argument("--sub-warmup", type=int, default=3)
    ap.add_argument("--sub-fp64-stride", type=int, default=4)
    ap.add_argument("--sub-requests", type=int, default=1000)
    ap.add_argument("--requests", type=int, default=10000)
    ap.add_argument("--serve-pool", type=int, default=1000)
    ap.add_argument("--capacity-requests", type=int, default=1000)
    ap.add_argument("--load", type=float, default=0.8)
    ap.add_argument("--iters-per-launch", type=int, default=1000000)
    # serve launch shape (measured on the 1,000-request mix: 1024 threads 6.6e6
    # DOF/s of capacity against 4.6e6 at 512; gang boost 16 keeps p50 lower than 4)
    ap.add_argument("--threads", type=int, default=1024)
    ap.add_argument("--gang-boost", type=int, default=16)
    ap.add_argument("--slice-us", type=int, default=40000, help="serve: time slice of a launch")
    ap.add_argument("--submit-threads", type=int, default=0)
    ap.add_argument("--serve-fp64-sample", type=int, default=200)
    # transient diffusion
    ap.add_argument("--heat-nx", type=int, default=256)
    ap.add_argument("--heat-nz", type=int, default=64)
    ap.add_argument("--heat-steps", type=int, default=100)
    ap.add_argument("--dt", type=float, default=1e-3)
    ap.add_argument("--heat-tol", type=float, default=1e-9)
    # residual replacement after a 1e3 fall of the FP32 residual: the mass
    # term keeps the step's system well conditioned, so two replacements per
    # step reach the tolerance in the same 164 inner iterations as four at 1e-2
    # (33.5 against 35.5 ms per step, solution error 2.3e-9)
    ap.add_argument("--heat-inner-tol", type=float, default=1e-3)
    ap.add_argument("--heat-reassemble", action="store_true", help="assemble C/dt + K every step")
    ap.add_argument("--cpu-heat-nx", type=int, default=48)
    args = ap.parse_args()
    if args.warmup < 3:
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    ref = args.impl == "reference"
    if args.config == "heat":
        out = run_heat_reference(args) if ref else run_heat(args)
    elif args.config == "batch":
        out = run_batch_reference(args) if ref else run_batch(args)
    elif args.config == "serve":
        out = run_serve_reference(args) if ref else run_serve(args)
    else:
        out = run_reference(args) if ref else run_ours(args)
    if out is not None:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
