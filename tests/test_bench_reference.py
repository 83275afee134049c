"""The bench's reference arm on the host: where the reference's own code was
compiled (oracle/_ref), the cube's reference figure comes from it -- the
whole system assembled once by its element code and Equations, and each step
two of its Equations::solve calls on that full system, stopped after a known
number of iterations -- and the product library is never loaded."""
import json
import os
import subprocess
import sys
from types import SimpleNamespace

import numpy as np
import pytest

from betanoox_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _need_ref(oracle):
    if not (oracle.RefLeaf.available() and oracle.RefEquations.available()):
        pytest.skip("oracle/_ref not built (reference tree absent)")


def test_eps_after_picks_a_first_crossing():
    sys.path.insert(0, ROOT)
    import bench
    tr = [10.0, 5.0, 6.0, 4.0, 3.0, 3.0, 1.0]
    assert bench._eps_after(tr, 2)[0] == 2
    assert bench._eps_after(tr, 3)[0] == 4          # 6.0 is not below 5.0
    assert bench._eps_after(tr, 6)[0] == 7          # 3.0 repeats: not below the earlier 3.0
    assert bench._eps_after(tr, 8) is None
    k, eps = bench._eps_after(tr, 4)
    assert all(v > eps for v in tr[:k - 1]) and tr[k - 1] < eps


@pytest.mark.parametrize("solver", ["parcg", "serial"])
def test_reference_cube_setup_and_step(oracle, solver):
    """The setup's bounded solve is checked against the oracle's iterate; a
    step gives a positive rate whose full solve covers the measured count."""
    _need_ref(oracle)
    sys.path.insert(0, ROOT)
    import bench
    m = W.cube_hex8(8, seed=2)
    args = SimpleNamespace(tol=1e-10, ref_iters_a=2, ref_iters_b=6, ref_solver=solver)
    R = bench.reference_cube_setup(m, args)
    assert R["check"] <= 1e-9 and R["kb"] > R["ka"] >= 2
    # the count is the oracle's full solve of the same system to ||r||/||b|| <= tol
    s = oracle.System(m)
    s.set_bc(m.restrained, m.prescribed, m.load)
    s.build_pattern()
    s.assemble(m.params, m.order)
    rc, x, st, _ = s.csr().pcg(s.rhs(), 1e-10, rule=oracle.Csr.RULE_RB, threads=2)
    assert rc == 0 and abs(st.iterations - R["iters_full"]) <= 2
    v, wall, t_it, t_fix = bench.reference_cube_step(R, m.ndof)
    R["rs"].close()
    assert v > 0 and wall > 0 and t_it > 0 and t_fix >= 0


def test_reference_arm_prints_one_json_line_without_the_product(oracle):
    """bench.py --impl reference on a small cube: standard output is exactly
    one JSON line (the reference code's own messages are kept off it), with
    the same config record as the GPU arm, and libbeta_gpu.so is never mapped
    into the process."""
    _need_ref(oracle)
    code = ("import sys; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '2', '--warmup', '1', "
            "'--n', '10']; import bench; bench.main(); "
            "maps = open('/proc/self/maps').read(); "
            "sys.stderr.write('PRODUCT_MAPPED=%d\\n' % ('libbeta_gpu' in maps))")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    assert len(lines) == 1, r.stdout
    assert "PRODUCT_MAPPED=0" in r.stderr
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["e2e"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] == 2
    sys.path.insert(0, ROOT)
    import bench
    args = SimpleNamespace(tol=1e-10, inner_tol=0.01)
    assert d["config"] == json.loads(json.dumps(bench.cube_config(W.cube_hex8(10), args, 1)))
    assert d["ms_per_step"] * d["steps"] < 60e3


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
