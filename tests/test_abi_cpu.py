"""The C ABI library without a GPU: it loads, exports every declared symbol,
and its host-side structure step is bit-exact with the oracle."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from betanoox_b200 import _abi
from betanoox_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    with open(os.path.join(ROOT, "include", "beta_gpu.h")) as f:
        src = f.read()
    return sorted(set(re.findall(r"BETA_GPU_API\s+(?:const\s+)?\w+\*?\s+\**(beta_gpu_\w+)\s*\(", src)))


def test_every_declared_symbol_is_exported(abi):
    names = _declared()
    assert len(names) >= 19
    for n in names:
        assert hasattr(abi, n), n
    assert set(names) == set(_abi.SIGNATURES), "binding table out of step with the header"


def test_version(abi):
    assert abi.beta_gpu_version() >= 10000


def _host_pattern(abi, m, rest=None):
    r = np.ascontiguousarray(m.restrained if rest is None else rest, np.uint8)
    conn = np.ascontiguousarray(m.conn, np.int32)
    fd = np.ascontiguousarray(m.first_dof, np.int32)
    nnz = C.c_longlong()
    st = abi.beta_gpu_pattern_lower_host(m.nnode, m.nelem, m.nnpe, m.ndpn, conn.ctypes.data, fd.ctypes.data,
                                         r.ctypes.data, C.byref(nnz), None, None)
    assert st == 0
    rp = np.zeros(m.ndof + 1, np.int64)
    col = np.zeros(nnz.value, np.int32)
    st = abi.beta_gpu_pattern_lower_host(m.nnode, m.nelem, m.nnpe, m.ndpn, conn.ctypes.data, fd.ctypes.data,
                                         r.ctypes.data, C.byref(nnz), rp.ctypes.data, col.ctypes.data)
    assert st == 0
    return rp, col


@pytest.mark.parametrize("make", [
    lambda: W.plate_quad4(9),
    lambda: W.cube_hex8(5, seed=1),
    lambda: W.heat_slab(6, 5, 4),
    lambda: W.rve_hex8(5, 17),
])
def test_host_pattern_bit_exact(abi, oracle, make):
    m = make()
    s = oracle.System(m)
    s.set_bc(m.restrained, m.prescribed, m.load)
    s.build_pattern()
    rp, col, _ = s.export_lower()
    rp2, col2 = _host_pattern(abi, m)
    np.testing.assert_array_equal(rp, rp2)
    np.testing.assert_array_equal(col, col2)


def test_host_pattern_ragged_restraints(abi, oracle):
    """Random restraint masks (partially restrained nodes) keep the pattern exact."""
    m = W.cube_hex8(4, seed=9)
    rng = np.random.default_rng(5)
    rest = (rng.uniform(size=m.ndof) < 0.3).astype(np.uint8)
    s = oracle.System(m)
    s.set_bc(rest, np.zeros(m.ndof), np.where(rest, 0.0, m.load))
    s.build_pattern()
    rp, col, _ = s.export_lower()
    rp2, col2 = _host_pattern(abi, m, rest)
    np.testing.assert_array_equal(rp, rp2)
    np.testing.assert_array_equal(col, col2)


def test_host_pattern_rejects_bad_numbering(abi):
    m = W.cube_hex8(2)
    conn = np.ascontiguousarray(m.conn, np.int32)
    fd = (np.arange(m.nnode, dtype=np.int32) * 3)[::-1].copy()
    r = np.zeros(m.ndof, np.uint8)
    nnz = C.c_longlong()
    st = abi.beta_gpu_pattern_lower_host(m.nnode, m.nelem, 8, 3, conn.ctypes.data, fd.ctypes.data, r.ctypes.data,
                                         C.byref(nnz), None, None)
    assert st == _abi.ERR_UNSUPPORTED


def test_create_without_gpu_fails_cleanly(abi):
    """On a machine without a CUDA device the context refuses to exist (no CPU fallback)."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("GPU present")
    except Exception:
        pass
    h = C.c_void_p()
    st = abi.beta_gpu_create(C.byref(h), 0)
    assert st != 0 and not h.value


def test_structured_block_count_matches_pattern():
    """The batch bench counts node-pair blocks of n^3 cubes as (3n+1)^3."""
    import bench
    for n in (1, 2, 5):
        m = W.rve_hex8(n, 3)
        assert bench.structured_nblk(m) == bench._nblk(m)


def test_serve_requests_cover_families_and_sizes():
    ms = [W.serve_request(5, i) for i in range(60)]
    fams = {m.meta["family"] for m in ms}
    assert fams == set(W.SERVE_FAMILIES)
    nd = np.array([m.ndof for m in ms])
    assert nd.min() >= 500 and nd.max() <= 6e5
    for m in ms[:6]:
        assert m.restrained.any() and np.isfinite(m.params).all()
