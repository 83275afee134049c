"""Bounded device waits: a gang barrier that cannot complete gives up after its
limit, the launch returns BETA_GPU_TIMEOUT, and the context stays usable.

The failure is made on the host: the plan gives the first gang a member that
is never launched (a flag that nothing sets), with a 20 ms limit.  Nothing
faults, traps or hangs.
"""
import ctypes as C

import numpy as np
import pytest

from betanoox_b200 import Batch, _abi, opts
from betanoox_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_gang_barrier_timeout_is_reported_and_recoverable(oracle):
    big = W.rve_hex8(16, 8)
    small = W.plate_quad4(10)
    b = Batch(hbm_budget=1 << 30)
    b.tune(512, 64)  # the big system forms a gang
    ids = [b.add(big), b.add(small)]
    assert b.lib.beta_gpu_batch_test_barrier(b.h, 20_000_000, 1) == _abi.OK
    with pytest.raises(_abi.BetaGpuError) as e:
        b.run(opts(tol=1e-12))
    assert e.value.status == _abi.TIMEOUT
    assert b.info()["gangs"] >= 1
    # the context is usable: normal limit, same systems, full solve
    assert b.lib.beta_gpu_batch_test_barrier(b.h, 2_000_000_000, 0) == _abi.OK
    assert b.run(opts(tol=1e-12)) == 0  # the interrupted system restarts by itself
    s = oracle.System(big)
    s.set_bc(big.restrained, big.prescribed, big.load)
    s.build_pattern()
    s.assemble(big.params, big.order)
    _, ut, _ = s.solve(eps=1e-14, maxit=300000)
    rc, u, st = b.result(ids[0])
    assert rc == _abi.OK and np.linalg.norm(u - ut) / np.linalg.norm(ut) <= 1e-8
