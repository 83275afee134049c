"""The bench's reference arm on the host: where the reference's own code was
compiled (oracle/_ref), the cube's reference figure comes from it -- element
B/addToKe, Equations pattern and addMatrix, and the faster of
SymmetricSparseMatrix::solve and the two-thread ParCG solve -- with the
oracle's all-core port beside it."""
import os
import sys
from types import SimpleNamespace

import pytest

from betanoox_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_code_baseline_times_the_reference(oracle):
    if not (oracle.RefLeaf.available() and oracle.RefEquations.available()):
        pytest.skip("oracle/_ref not built (reference tree absent)")
    sys.path.insert(0, ROOT)
    import bench
    m = W.cube_hex8(6, seed=2)
    args = SimpleNamespace(cpu_elems=64, cpu_ref_n=4, cpu_ref_eps=1e-6)
    cb = bench.reference_code_baseline(m, args, 100)
    assert cb["kind"] == "reference" and cb["cores"] in (1, 2)
    assert cb["value"] > 0 and cb["seconds_full_solve_est"] > 0
    assert "SymmetricSparseMatrix::solve" in cb["sample"] and "ParCGMatrix::solve" in cb["sample"]


def test_reference_arm_prints_one_json_line():
    """bench.py --impl reference on a small cube: standard output is exactly
    one JSON line (the reference code's own messages are kept off it), with
    the reference's figure and, where oracle/_ref exists, the port beside it."""
    import json
    import subprocess
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0", "--n", "12", "--cpu-elems", "500", "--cpu-ref-n", "6", "--cpu-n", "8",
                        "--cpu-iters", "5"], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["e2e"]["value"] == d["value"]
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port")
    if cb["kind"] == "reference":
        assert cb["port_all_cores"]["kind"] == "port"


def test_reference_full_solves_run_the_reference(oracle):
    """The batch arm's sampler: whole RVEs solved by the reference's own code
    after the port, both timed on the same systems."""
    if not (oracle.RefLeaf.available() and oracle.RefEquations.available()):
        pytest.skip("oracle/_ref not built (reference tree absent)")
    sys.path.insert(0, ROOT)
    import bench
    models = [W.rve_hex8(4, seed=3), W.rve_hex8(5, seed=4)]
    n, d, t_ref, t_port = bench.reference_full_solves(models, 1e-8, 1e9, 2)
    assert n == 2 and d == sum(m.ndof for m in models) and t_ref > 0 and t_port > 0


def test_reference_heat_baseline_runs_the_reference(oracle):
    """The heat arm's sampler: transient steps by the reference's own element
    step terms, Equations scatter and solve, after the oracle's step."""
    if not (oracle.RefLeaf.available() and oracle.RefEquations.available()):
        pytest.skip("oracle/_ref not built (reference tree absent)")
    sys.path.insert(0, ROOT)
    import bench
    args = SimpleNamespace(cpu_heat_nx=8, heat_nz=4, heat_nx=16, dt=1e-3, heat_tol=1e-10)
    cb = bench.reference_heat_baseline(args, W.heat_slab(16, 16, 4, order=2))
    assert cb["kind"] == "reference" and cb["value"] > 0 and cb["port_single_thread"]["value"] > 0


def test_reference_full_solves_cover_the_serve_kinds(oracle):
    """The sampler on one small request of each serving kind (quad4 plane
    stress, hex8 elasticity, hex8 steady diffusion)."""
    if not (oracle.RefLeaf.available() and oracle.RefEquations.available()):
        pytest.skip("oracle/_ref not built (reference tree absent)")
    sys.path.insert(0, ROOT)
    import bench
    picked = {}
    for j in range(60):
        m = W.serve_request(11, j, dof_lo=300.0, dof_hi=3000.0)
        picked.setdefault(m.kind, m)
        if len(picked) == 3:
            break
    assert sorted(picked) == [1, 2, 3]
    models = list(picked.values())
    n, d, t_ref, t_port = bench.reference_full_solves(models, 1e-8, 1e9, 2)
    assert n == 3 and d == sum(m.ndof for m in models)
