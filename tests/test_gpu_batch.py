"""Batched persistent solves: every system's answer equals its own solve.

Each system in a batch is checked against the FP64 oracle solution (1e-8
relative L2, the mixed-precision contract), and a batch advanced in short
launches (the serving loop's preemption) must give bit-identical iterates to
one uninterrupted launch.
"""
import numpy as np
import pytest

from betanoox_b200 import Batch, _abi, opts
from betanoox_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _truth(oracle, m):
    s = oracle.System(m)
    assert s.set_bc(m.restrained, m.prescribed, m.load) == 0
    s.build_pattern()
    assert s.assemble(m.params, m.order) == 0
    rc, u, _ = s.solve(eps=1e-14, maxit=300000)
    return u


def _steady_heat(n=6):
    m = W.heat_slab(n, n, n // 2 + 2, order=2)
    pres = np.zeros(m.ndof)
    pres[np.isclose(m.xyz[:, 0], 0.0)] = 1.0  # T = 1 on x = 0, T = 0 on the other faces
    m.prescribed = pres
    return m


def _mix():
    return [W.rve_hex8(6, 1), W.cube_hex8(5, seed=2), W.plate_quad4(10), _steady_heat(6), W.rve_hex8(8, 3),
            W.plate_quad4(7, E=2e4)]


def test_batch_each_system_matches_oracle(oracle):
    models = _mix()
    b = Batch(hbm_budget=1 << 30)
    ids = [b.add(m) for m in models]
    assert b.run(opts(tol=1e-12)) == 0
    for sid, m in zip(ids, models):
        rc, u, st = b.result(sid)
        assert rc == _abi.OK, st.as_dict()
        ut = _truth(oracle, m)
        assert np.linalg.norm(u - ut) / np.linalg.norm(ut) <= 1e-8, (m.name, st.as_dict())


def test_batch_short_launches_equal_one_launch():
    models = _mix()
    b1 = Batch(hbm_budget=1 << 30)
    ids1 = [b1.add(m) for m in models]
    b1.run(opts(tol=1e-12))
    b2 = Batch(hbm_budget=1 << 30)
    ids2 = [b2.add(m) for m in models]
    launches = 0
    while b2.run(opts(tol=1e-12), iters_per_launch=7) > 0:
        launches += 1
        assert launches < 10000
    assert launches > 1
    for i1, i2 in zip(ids1, ids2):
        _, u1, s1 = b1.result(i1)
        _, u2, s2 = b2.result(i2)
        assert s1.iterations == s2.iterations
        np.testing.assert_array_equal(u1, u2)


def test_batch_admission_by_budget_and_reuse():
    small = W.rve_hex8(6, 4)
    b = Batch(hbm_budget=24 << 20)  # room for only a few small systems
    ids = []
    while True:
        sid = b.add(small, raise_on_reject=False)
        if sid is None:
            break
        ids.append(sid)
        assert len(ids) < 1000
    assert len(ids) >= 1
    info = b.info()
    assert info["used"] <= info["pool"]
    b.remove(ids[0])
    assert b.add(small, raise_on_reject=False) is not None  # freed memory is reused


def test_batch_autotune_keeps_results(oracle):
    models = _mix()[:3]
    b = Batch(hbm_budget=1 << 30)
    ids = [b.add(m) for m in models]
    t, g = b.autotune(opts(tol=1e-12), budget=10)
    assert t in (256, 512, 1024) and 0 <= g <= 64
    assert b.run(opts(tol=1e-12)) == 0
    for sid, m in zip(ids, models):
        rc, u, st = b.result(sid)
        ut = _truth(oracle, m)
        assert rc == _abi.OK and np.linalg.norm(u - ut) / np.linalg.norm(ut) <= 1e-8


def test_add_many_equals_add_and_reset_repeats():
    models = _mix()
    b1 = Batch(hbm_budget=1 << 30)
    ids1 = [b1.add(m) for m in models]
    b2 = Batch(hbm_budget=1 << 30)
    ids2 = b2.add_many(models, host_threads=4)
    assert b1.run(opts(tol=1e-12)) == 0 and b2.run(opts(tol=1e-12)) == 0
    first = [b2.result(i)[1] for i in ids2]
    for i1, i2 in zip(ids1, ids2):
        np.testing.assert_array_equal(b1.result(i1)[1], b2.result(i2)[1])
    assert b2.info()["last_launch_ns"] > 0
    b2.reset()  # same systems again, re-assembled from the pool
    assert b2.run(opts(tol=1e-12)) == 0
    for i2, u in zip(ids2, first):
        np.testing.assert_array_equal(b2.result(i2)[1], u)


def test_result_independent_of_gang_size_and_cta_size():
    """Fixed-order sums: one CTA, a gang of any size, or another CTA size give
    bit-identical iterates."""
    models = [W.rve_hex8(12, 5), W.plate_quad4(40), _steady_heat(10)]
    out = []
    for threads, boost in [(512, 0), (512, 64), (256, 16), (1024, 2)]:
        b = Batch(hbm_budget=1 << 30)
        b.tune(threads, boost)
        ids = [b.add(m) for m in models]
        assert b.run(opts(tol=1e-12), iters_per_launch=0) == 0
        if boost == 64:
            assert b.info()["gangs"] >= 1
        out.append([(b.result(i)[2].iterations, b.result(i)[1]) for i in ids])
        b.close()
    for other in out[1:]:
        for (i0, u0), (i1, u1) in zip(out[0], other):
            assert i0 == i1
            np.testing.assert_array_equal(u0, u1)


def test_time_sliced_launches_equal_one_launch():
    """Launches cut by a time slice -- gangs and single CTAs, FP32 and FP64
    modes -- give the iterates of one uninterrupted launch."""
    models = [W.rve_hex8(12, 5), W.plate_quad4(40), _steady_heat(10), W.rve_hex8(6, 1), W.plate_quad4(7, E=2e4)]

    def solve(slice_us):
        b = Batch(hbm_budget=1 << 30)
        b.tune(512, 64)
        b.set_switch(30)
        b.set_slice(slice_us)
        ids = [b.add(m) for m in models]
        launches = 1
        while b.run(opts(tol=1e-12)) > 0:
            launches += 1
            assert launches < 20000
        out = []
        for i in ids:
            rc, u, st = b.result(i)
            assert rc == _abi.OK, st.as_dict()
            out.append((st.iterations, st.reserved, u))
        b.close()
        return launches, out

    n1, ref = solve(0)
    n2, cut = solve(300)
    assert n1 == 1 and n2 > 3
    assert any(r for _, r, _ in ref)  # some system went on in FP64
    for (i0, r0, u0), (i1, r1, u1) in zip(ref, cut):
        assert i0 == i1 and r0 == r1
        np.testing.assert_array_equal(u0, u1)


def test_fp64_switch_matches_oracle_and_is_mix_independent(oracle):
    """A system whose FP32 cycles are long continues as FP64 matrix-free PCG;
    its answer still meets the oracle and does not depend on the mix."""
    plate = W.serve_request(99, 46)  # slender quad4 plate (~64k dofs, slow FP32 cycles)
    small = W.plate_quad4(12)
    models = [plate, W.rve_hex8(6, 1), small]
    b = Batch(hbm_budget=1 << 30)
    b.set_switch(40)
    ids = [b.add(m) for m in models]
    assert b.run(opts(tol=1e-12)) == 0
    rc, u, st = b.result(ids[0])
    assert rc == _abi.OK and st.reserved == 1, st.as_dict()
    ut = _truth(oracle, plate)
    assert np.linalg.norm(u - ut) / np.linalg.norm(ut) <= 1e-8
    b1 = Batch(hbm_budget=1 << 30)
    b1.set_switch(40)
    i1 = b1.add(plate)
    assert b1.run(opts(tol=1e-12), iters_per_launch=37) >= 0
    while b1.run(opts(tol=1e-12), iters_per_launch=37) > 0:
        pass
    rc1, u1, st1 = b1.result(i1)
    assert st1.iterations == st.iterations
    np.testing.assert_array_equal(u, u1)
