"""Host structure build reused by a solver context (HostPattern::keep_scratch):
a pattern rebuilt into the memory of an earlier, different mesh equals a
fresh build in every field, and so does a single-threaded build; the node
rows and the element slot map equal their definition built the plain way; the
column-run layout of the FP32 block matrix places every block in its run
(tests/cpp/pattern_reuse_check.cpp, compiled here against the host sources;
no GPU needed)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(tmp_path, name, extra):
    exe = os.path.join(str(tmp_path), name)
    subprocess.run(["g++", "-std=c++17", "-O2", "-pthread", "-Wall", *extra,
                    os.path.join(ROOT, "tests", "cpp", "pattern_reuse_check.cpp"),
                    os.path.join(ROOT, "betanoox_b200", "csrc", "pattern.cpp"), "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count(" equal") == 8
    # rows and slot map against their definition, built the plain way
    assert r.stdout.count(" as defined") == 8 and "NOT AS DEFINED" not in r.stdout
    assert r.stdout.count(" valid") == 8 and "INVALID" not in r.stdout
    # the 70^3 grid with one dof per node takes the compact form of its runs
    assert any("hex8 n=70 nd=1" in line and "compact=1" in line for line in r.stdout.splitlines())
    # lexicographic hex8 grids and the quad4 plate take runs of 3; the
    # shuffled numberings keep one column per block
    runs = dict(line[5:].rsplit(" run=", 1) for line in r.stdout.splitlines() if line.startswith("runs "))
    for name, tail in runs.items():
        want = "1" if "shuffled" in name else "3"
        assert tail.split()[0] == want, (name, tail)
    assert "NOT REFUSED" not in r.stdout and r.stdout.count("refused") == 1
    return [line for line in r.stdout.splitlines() if line.startswith("hash ")]


def test_reused_pattern_equals_fresh_build(tmp_path):
    """Also: the node-graph passes' bandwidth-sized marker form (used when
    node-sized markers would exceed their memory budget) and their
    sort-per-row form (a span too wide even for that) build the same pattern,
    field for field, as the node-sized form."""
    default = _run(tmp_path, "pattern_reuse_check", [])
    bounded = _run(tmp_path, "pattern_reuse_check_bounded", ["-DBETA_PATTERN_MARK_BUDGET=0"])
    sorted_rows = _run(tmp_path, "pattern_reuse_check_sorted", ["-DBETA_PATTERN_MARK_BUDGET=0",
                                                                  "-DBETA_PATTERN_SPAN_CAP=0"])
    assert len(default) == 16 and default == bounded == sorted_rows
