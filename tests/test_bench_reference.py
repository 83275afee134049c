"""The bench's reference arm on the host: where the reference's own code was
compiled (oracle/_ref), the cube's reference figure comes from it -- element
B/addToKe, Equations pattern and addMatrix, SymmetricSparseMatrix::solve --
serially, with the oracle's all-core port beside it."""
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
    assert cb["kind"] == "reference" and cb["cores"] == 1
    assert cb["value"] > 0 and cb["seconds_full_solve_est"] > 0
    assert "SymmetricSparseMatrix::solve" in cb["sample"]
