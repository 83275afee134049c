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


@pytest.mark.parametrize("make", [lambda: W.plate_quad4(4), lambda: W.cube_hex8(3, seed=7),
                                  lambda: W.heat_slab(4, 3, 3)])
def test_host_pattern_unused_free_node(abi, oracle, make):
    """A node no element uses, its dofs left free: Equations gives each of its
    (empty) rows the diagonal alone -- no entries between its own dofs."""
    import dataclasses
    m = W.renumbered(make(), 2, unused_node=True)
    r = m.restrained.copy()
    r[-m.ndpn:] = 0
    m = dataclasses.replace(m, restrained=r)
    s = oracle.System(m)
    s.set_bc(m.restrained, m.prescribed, m.load)
    s.build_pattern()
    rp, col, _ = s.export_lower()
    rp2, col2 = _host_pattern(abi, m)
    np.testing.assert_array_equal(rp, rp2)
    np.testing.assert_array_equal(col, col2)
    for r in range(m.ndof - m.ndpn, m.ndof):
        assert list(col2[rp2[r]:rp2[r + 1]]) == [r]


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


def _plan(abi, work, slices, ctas=148, threads=512, boost=4):
    n = len(work)
    w = (C.c_longlong * max(1, n))(*work)
    s = (C.c_int * max(1, n))(*slices)
    g = (C.c_int * max(1, n))()
    ng = abi.beta_gpu_gang_plan(n, w, s, ctas, threads, boost, g)
    return ng, list(g)[:max(0, ng)]


def test_gang_plan_single_system_takes_the_gpu(abi):
    ng, g = _plan(abi, [10 ** 8], [100000])
    assert ng == 1 and g == [148]
    ng, g = _plan(abi, [10 ** 6], [200])  # capped: every warp keeps two slices
    assert ng == 1 and g == [200 // 32]
    assert _plan(abi, [10 ** 8], [100000], boost=0)[0] == 0


def test_gang_plan_invariants_on_random_batches(abi):
    rng = np.random.default_rng(3)
    for _ in range(200):
        n = int(rng.integers(1, 600))
        sl = np.sort(rng.integers(1, 8000, size=n))[::-1]
        work = sl.astype(np.int64) * 27 * 32 * 9
        ctas = int(rng.integers(2, 300))
        boost = int(rng.choice([0, 1, 2, 4, 8, 64]))
        ng, g = _plan(abi, work.tolist(), sl.tolist(), ctas=ctas, boost=boost)
        assert 0 <= ng <= min(n, ctas // 2)
        assert sum(g) <= ctas and all(x >= 2 for x in g)
        assert all(g[i] >= g[i + 1] for i in range(len(g) - 1))
        for i, x in enumerate(g):
            assert x <= max(2, sl[i] // 32)


def test_gang_plan_rejects_unsorted_input(abi):
    assert _plan(abi, [5, 9], [10, 10])[0] == -_abi.ERR_ARG
