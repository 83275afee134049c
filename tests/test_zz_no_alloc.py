"""The allocation-free PCG entry point against the allocating one.

beta_gpu_csr_pcg_device_noalloc exists for callers that cannot let a library
call cudaMalloc (an application that has handed HBM to its own pool, or that
cannot afford the device-wide synchronisation cudaMalloc/cudaFree imply): its
scratch is a fixed array inside the library.  Two calls in a row must give the
allocating entry point's answer -- the second call finds the first call's
leftovers in the shared array and must clear what has to start at zero.

This file is collected last on purpose, and runs alone as well.
"""
import ctypes as C

import numpy as np
import pytest

from betanoox_b200 import _abi
from betanoox_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _device_system(oracle, m):
    import torch
    import scipy.sparse as sp
    s = oracle.System(m)
    s.set_bc(m.restrained, m.prescribed, m.load)
    s.build_pattern()
    s.assemble(m.params, m.order)
    rp, col, val = s.export_lower()
    n = m.ndof
    rows = np.repeat(np.arange(n), np.diff(rp))
    L = sp.csr_matrix((val, (rows, col)), shape=(n, n))
    A = (L + sp.triu(L.T, 1)).tocsr()
    A.sort_indices()
    dev = torch.device("cuda:0")
    t = dict(
        rp=torch.tensor(A.indptr.astype(np.int32), device=dev),
        ci=torch.tensor(A.indices.astype(np.int32), device=dev),
        v=torch.tensor(A.data, device=dev, dtype=torch.float64),
        b=torch.tensor(s.rhs(), device=dev, dtype=torch.float64),
    )
    return n, t


def _solve(fn, n, t, tol=1e-12):
    import torch
    x = torch.zeros(n, device="cuda:0", dtype=torch.float64)
    st = _abi.SolveStats()
    torch.cuda.synchronize()
    rc = fn(n, t["rp"].data_ptr(), t["ci"].data_ptr(), t["v"].data_ptr(), t["b"].data_ptr(), x.data_ptr(),
            _abi.STOP_RB, tol, 100000, None, C.byref(st))
    torch.cuda.synchronize()
    return rc, x.cpu().numpy(), st


def test_noalloc_matches_allocating_solver_twice(oracle):
    lib = _abi.load()
    for m in (W.cube_hex8(7, seed=21), W.plate_quad4(16)):
        n, t = _device_system(oracle, m)
        rc0, x0, st0 = _solve(lib.beta_gpu_csr_pcg_device, n, t)
        assert rc0 == _abi.OK
        for _ in range(2):  # two calls in a row share the same scratch array
            rc, x, st = _solve(lib.beta_gpu_csr_pcg_device_noalloc, n, t)
            assert rc == _abi.OK, st.as_dict()
            assert np.linalg.norm(x - x0) <= 1e-12 * np.linalg.norm(x0)
            assert st.iterations == st0.iterations
            assert st.true_rel_residual <= 1e-11


def test_noalloc_larger_then_smaller_system(oracle):
    """A smaller system right after a larger one: the shared array still holds
    the larger system's vectors past the smaller one's n, and a different grid
    size leaves other reduction partials behind.  Both answers must equal the
    allocating solver's."""
    lib = _abi.load()
    big, small = W.cube_hex8(8, seed=5), W.plate_quad4(10)
    nb, tb = _device_system(oracle, big)
    ns, ts = _device_system(oracle, small)
    assert nb > 4 * ns
    ref = {}
    for key, (n, t) in (("big", (nb, tb)), ("small", (ns, ts))):
        rc0, x0, st0 = _solve(lib.beta_gpu_csr_pcg_device, n, t)
        assert rc0 == _abi.OK
        ref[key] = (x0, st0.iterations)
    # no allocating call between the two allocation-free ones
    got = {}
    for key, (n, t) in (("big", (nb, tb)), ("small", (ns, ts))):
        rc, x, st = _solve(lib.beta_gpu_csr_pcg_device_noalloc, n, t)
        assert rc == _abi.OK, st.as_dict()
        got[key] = (x, st.iterations)
    for key in ("big", "small"):
        x0, it0 = ref[key]
        x, it = got[key]
        assert np.linalg.norm(x - x0) <= 1e-12 * np.linalg.norm(x0), key
        assert it == it0, key


def test_noalloc_bad_arguments_report_status():
    lib = _abi.load()
    st = _abi.SolveStats()
    st.status = 12345
    rc = lib.beta_gpu_csr_pcg_device_noalloc(0, None, None, None, None, None, _abi.STOP_RB, 1e-10, 10, None,
                                             C.byref(st))
    assert rc == _abi.ERR_ARG
    assert st.status == _abi.ERR_ARG


def test_noalloc_rejects_oversized_systems():
    import torch
    lib = _abi.load()
    tiny = torch.zeros(4, device="cuda:0", dtype=torch.float64)
    ti = torch.zeros(4, device="cuda:0", dtype=torch.int32)
    st = _abi.SolveStats()
    rc = lib.beta_gpu_csr_pcg_device_noalloc(_abi.NOALLOC_MAX_ROWS + 1, ti.data_ptr(), ti.data_ptr(),
                                             tiny.data_ptr(), tiny.data_ptr(), tiny.data_ptr(), _abi.STOP_RB,
                                             1e-10, 10, None, C.byref(st))
    assert rc == _abi.ERR_TOO_LARGE
