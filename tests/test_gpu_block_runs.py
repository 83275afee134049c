"""The FP32 node-block matrix with one column index per run of up to three
consecutive node columns (what a solver context builds by default where it
makes the matrix at least 5 % smaller) against one column index per block,
on the GPU.  The runs visit the blocks of a row in the same ascending column
order and add exact zeros between them, so the two layouts must agree bit
for bit: the assembled FP32 values, the SpMV, the mixed-precision solve
(iterations and solution), the transient steps and the mixed Newton loop.
Both layouts are checked against the oracle by the parity tests through the
default context; here a renumbered mesh also shows that a numbering without
runs keeps one index per block.
"""
import numpy as np
import pytest

from betanoox_b200 import BetaGpuError, Solver, _abi, opts
from betanoox_b200 import workloads as W

pytestmark = pytest.mark.gpu

MODELS = {
    "hex8": lambda: W.cube_hex8(10, seed=3),          # 3 dofs per node
    "quad4": lambda: W.plate_quad4(40),               # 2 dofs per node
    "heat": lambda: W.heat_slab(12, 10, 6, order=3),  # 1 dof per node
    "rve": lambda: W.rve_hex8(9, 4),
    # x-rows of 97 nodes: most 32-node slices lie inside one row, so the runs
    # take their compact form (one offset per run for such a slice)
    "heat_long": lambda: W.heat_slab(96, 10, 6, order=3),
}


def _pair(m):
    out = []
    for run in (1, 3):
        g = Solver()
        g.set_block_runs(run)
        g.load_model(m)
        g.build_pattern()
        out.append(g)
    return out


@pytest.mark.parametrize("name", list(MODELS))
def test_runs_equal_one_column_per_block(name):
    m = MODELS[name]()
    g1, g3 = _pair(m)
    l1, l3 = g1.block_layout(), g3.block_layout()
    assert l1[0] == 1 and l3[0] == 3
    assert l3[3] <= 0.95 * l1[3]
    if name == "heat_long":
        assert l3[4] == 1 and l3[3] <= 0.9 * l1[3]
    g1.assemble(_abi.FP32)
    g3.assemble(_abi.FP32)
    v1, _ = g1.lower_values(_abi.FP32)
    v3, _ = g3.lower_values(_abi.FP32)
    np.testing.assert_array_equal(v1, v3)
    x = np.random.default_rng(1).standard_normal(m.ndof)
    np.testing.assert_array_equal(g1.matvec(x, _abi.FP32), g3.matvec(x, _abi.FP32))
    for precond in (_abi.PRECOND_BLOCK_JACOBI, _abi.PRECOND_JACOBI):
        o = opts(mode=_abi.MODE_MPIR, precond=precond, tol=1e-10)
        rc1, st1 = g1.solve(o)
        rc3, st3 = g3.solve(o)
        assert rc1 == rc3 == _abi.OK
        assert (st1.iterations, st1.outer_iterations) == (st3.iterations, st3.outer_iterations)
        np.testing.assert_array_equal(g1.download(), g3.download())


def test_runs_equal_in_transient_steps():
    m = W.heat_slab(10, 8, 6, order=3)
    g1, g3 = _pair(m)
    res = []
    for g in (g1, g3):
        g.heat_set_state(m.meta["u0"])
        st, tot = g.heat_run(1e-3, 3, opts(mode=_abi.MODE_MPIR, tol=1e-13, inner_tol=0.01, check_every=4))
        res.append((tot, g.heat_get_state()))
    assert res[0][0] == res[1][0]
    np.testing.assert_array_equal(res[0][1], res[1][1])


def test_runs_equal_in_mixed_newton():
    m = W.cantilever_hex8(nx=16, ny=2, nz=2, load=12.0)
    g1, g3 = _pair(m)
    out = []
    for g in (g1, g3):
        rc, st, hist = g.newton(opts(mode=_abi.MODE_MPIR, precond=_abi.PRECOND_BLOCK_JACOBI, inner_tol=1e-4,
                                     maxit=100000), max_residual=1e-10, max_newton=60)
        assert rc == _abi.OK
        out.append((st.iterations, st.linear_iterations, hist, g.download()))
    assert out[0][:2] == out[1][:2]
    np.testing.assert_array_equal(out[0][2], out[1][2])
    np.testing.assert_array_equal(out[0][3], out[1][3])


def test_numbering_without_runs_keeps_one_column_per_block():
    m = W.renumbered(W.cube_hex8(8, seed=5), seed=9)
    g = Solver()
    g.load_model(m)
    g.build_pattern()
    assert g.block_layout()[0] == 1
    g.set_block_runs(1)  # dropping the pattern: it must be built again
    with pytest.raises(BetaGpuError):
        g.block_layout()
