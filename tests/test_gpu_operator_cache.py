"""The FP64 hex8 diffusion operator from cached element matrices (K_e and
M_e integrated once per mesh and material set) against the same operator
integrated at every use, on the GPU: the operator, the transient steps in
FP64 and mixed precision and a steady mixed-precision solve agree to
rounding, and the cache follows material changes.  The oracle checks of the
heat paths (test_gpu_parity.py) run with the cache, the default."""
import dataclasses

import numpy as np
import pytest

from betanoox_b200 import Solver, _abi, opts
from betanoox_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _solver(m, cache):
    g = Solver()
    g.set_operator_cache(cache)
    g.load_model(m)
    g.build_pattern()
    return g


@pytest.mark.parametrize("mode", [_abi.MODE_FP64, _abi.MODE_MPIR])
def test_cached_operator_in_transient_steps(mode):
    m = W.heat_slab(12, 9, 7, order=2)
    out = []
    for cache in (False, True):
        g = _solver(m, cache)
        g.heat_set_state(m.meta["u0"])
        st, tot = g.heat_run(1e-3, 4, opts(mode=mode, tol=1e-12, inner_tol=0.01, check_every=4))
        out.append(g.heat_get_state())
    assert np.linalg.norm(out[1] - out[0]) <= 1e-12 * np.linalg.norm(out[0])


def test_cached_operator_in_steady_solve_and_after_a_material_change():
    m = W.heat_slab(10, 8, 6, order=3)
    # a heat input on the free nodes (the slab's faces are held at T = 0)
    q = np.random.default_rng(4).uniform(0.5, 1.5, m.ndof) * (np.asarray(m.restrained) == 0)
    m = dataclasses.replace(m, load=q)
    res = []
    for cache in (False, True):
        g = _solver(m, cache)
        g.assemble(_abi.FP32)
        rc, st = g.solve(opts(mode=_abi.MODE_MPIR, tol=1e-11))
        assert rc == _abi.OK
        u1 = g.download()
        # new conductivities: the cached matrices must be rebuilt
        p2 = np.array(m.params, copy=True)
        p2[:, :3] *= 1.7
        g.load_materials(p2)
        g.assemble(_abi.FP32)
        rc, st = g.solve(opts(mode=_abi.MODE_MPIR, tol=1e-11))
        assert rc == _abi.OK
        res.append((u1, g.download()))
    for a, b in zip(res[0], res[1]):
        assert np.linalg.norm(b - a) <= 1e-9 * np.linalg.norm(a)
    assert np.linalg.norm(res[1][1] - res[1][0]) > 1e-3 * np.linalg.norm(res[1][0])
