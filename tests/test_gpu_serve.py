"""Continuous-batching server: each result is the same alone and in the mix.

Requests arrive while others are being solved, join between bounded launches
and leave when they converge.  Every served solution must be bit-identical to
the same system served alone (same launch shape), and within 1e-8 relative L2
of the FP64 oracle solution (the mixed-precision contract).
"""
import threading
import time

import numpy as np
import pytest

from betanoox_b200 import Server, _abi, opts
from betanoox_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _truth(oracle, m):
    s = oracle.System(m)
    assert s.set_bc(m.restrained, m.prescribed, m.load) == 0
    s.build_pattern()
    assert s.assemble(m.params, m.order) == 0
    rc, u, _ = s.solve(eps=1e-14, maxit=300000)
    return u


def _mix():
    return [W.rve_hex8(6, 1), W.cube_hex8(5, seed=2), W.plate_quad4(10), W.rve_hex8(8, 3), W.rve_hex8(7, 9),
            W.plate_quad4(7, E=2e4), W.rve_hex8(5, 12), W.cube_hex8(4, seed=5)]


def _alone(m, **kw):
    with Server(o=opts(tol=TOL), **kw) as s:
        rid = s.submit(m)
        state, u, st, lat = s.wait(rid)
        assert state == _abi.REQ_DONE and st.status == _abi.OK, st.as_dict()
        return u, st


@pytest.mark.parametrize("kw", [dict(iters_per_launch=25, threads=512, gang_boost=4),
                                dict(iters_per_launch=100000, threads=512, gang_boost=16, slice_us=400)],
                         ids=["budget", "slice"])
def test_served_mix_equals_each_alone_and_oracle(oracle, kw):
    models = _mix()
    solo = [_alone(m, **kw) for m in models]
    with Server(hbm_budget=1 << 30, o=opts(tol=TOL), **kw) as s:
        rids = [None] * len(models)

        def arrivals():  # staggered arrivals: later requests join a running batch
            rng = np.random.default_rng(7)
            for i, m in enumerate(models):
                rids[i] = s.submit(m)
                time.sleep(float(rng.exponential(0.003)))

        t = threading.Thread(target=arrivals)
        t.start()
        t.join()
        out = [s.wait(r) for r in rids]
        stats = s.stats()
    assert stats["done"] == len(models) and stats["failed"] == 0 and stats["rejected"] == 0
    assert stats["launches"] >= 2
    for m, (u1, s1), (state, u2, s2, lat) in zip(models, solo, out):
        assert state == _abi.REQ_DONE and s2.status == _abi.OK, (m.name, s2.as_dict())
        assert lat > 0
        assert s1.iterations == s2.iterations
        np.testing.assert_array_equal(u1, u2)
        ut = _truth(oracle, m)
        assert np.linalg.norm(u2 - ut) / np.linalg.norm(ut) <= 1e-8, m.name


def test_queue_waits_for_pool_memory_and_rejects_oversize():
    small = W.rve_hex8(6, 4)
    big = W.rve_hex8(16, 4)
    with Server(hbm_budget=3 << 19, o=opts(tol=1e-10), iters_per_launch=20) as s:  # room for 2-3 small systems
        rids = [s.submit(small) for _ in range(8)]
        rbig = s.submit(big)
        states = [s.wait(r)[0] for r in rids]
        state_big = s.wait(rbig)[0]
        stats = s.stats()
    assert all(x == _abi.REQ_DONE for x in states)
    assert state_big == _abi.REQ_REJECTED
    assert stats["rejected"] == 1 and stats["done"] == 8
    assert stats["pool_used"] == 0


def test_cancel_and_bad_input():
    m = W.rve_hex8(8, 2)
    with Server(hbm_budget=1 << 30, o=opts(tol=1e-12), iters_per_launch=5) as s:
        rids = [s.submit(m) for _ in range(4)]
        s.cancel(rids[-1])
        states = [s.wait(r)[0] for r in rids]
        bad = W.cube_hex8(3)
        bad.xyz = bad.xyz.copy()
        bad.xyz[0, 0] = np.inf
        with pytest.raises(_abi.BetaGpuError) as e:
            s.submit(bad)
        assert e.value.status == _abi.ERR_NOT_FINITE
        with pytest.raises(_abi.BetaGpuError):
            s.poll(10 ** 9)
    assert states[:3] == [_abi.REQ_DONE] * 3
    assert states[3] in (_abi.REQ_CANCELLED, _abi.REQ_DONE)


def test_arrival_ends_the_running_slice():
    """Continuous batching under a long time slice: a small request that
    arrives while a big one is being solved is admitted during the running
    launch, which then ends its slice early (after at most one iteration past
    the 2 ms minimum), so the small request finishes long before the big one
    instead of waiting for the launch -- here, for the big solve -- to end."""
    big = W.cube_hex8(80, seed=3)  # 1.6 M dofs: a solve of a few hundred ms
    small = W.plate_quad4(8)
    with Server(hbm_budget=4 << 30, o=opts(tol=1e-10), iters_per_launch=10 ** 6, slice_us=20_000_000) as s:
        rb = s.submit(big)
        t_end = time.monotonic() + 60
        while s.poll(rb)[0] != _abi.REQ_RUNNING and time.monotonic() < t_end:
            time.sleep(0.002)
        time.sleep(0.02)  # the big system's launch is under way
        rs = s.submit(small)
        st_s, _, ss, lat_s = s.wait(rs)
        st_b, _, sb, lat_b = s.wait(rb)
        launches = s.stats()["launches"]
    assert st_s == st_b == _abi.REQ_DONE and ss.status == sb.status == _abi.OK
    assert lat_s < 0.5 * lat_b, (lat_s, lat_b)
    assert launches >= 2
