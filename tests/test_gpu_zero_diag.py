"""ReplaceZeroDiagonal on the GPU (LargeMatrix::CheckAndFixZeroDiagonal,
largeMatrix.cpp:43-79, set by the ReplaceZeroDiagonal command,
equation.cpp:1819-1823): the rows of a node no element uses hold only a zero
diagonal.  Without the option the solve is refused, as the reference exits;
with it, the plain FP64 and the mixed-precision solves give the oracle's
solution, whose replacement is pinned bit-identical against the reference's
own Equations solve (tests/test_oracle_pins.py)."""
import dataclasses

import numpy as np
import pytest

from betanoox_b200 import Solver, _abi, opts
from betanoox_b200 import workloads as W

pytestmark = pytest.mark.gpu

VALUE = 2.5  # the replacement value of the reference-pinned golden case


def _unused_node_model(base):
    m = W.renumbered(base, 2, unused_node=True)
    r = m.restrained.copy()
    r[-m.ndpn:] = 0  # the appended node's dofs left free: zero rows
    return dataclasses.replace(m, restrained=r)


@pytest.mark.parametrize("base", [lambda: W.plate_quad4(4), lambda: W.cube_hex8(3, seed=7)], ids=["quad4", "hex8"])
def test_zero_diagonal_refused_then_replaced(oracle, base):
    m = _unused_node_model(base())
    s = oracle.System(m)
    s.set_bc(m.restrained, m.prescribed, m.load)
    s.build_pattern()
    s.assemble(m.params, m.order)
    assert s.solve(eps=1e-10, maxit=10000)[0] == oracle.ERR_ZERO_DIAG
    s.set_zero_diag(VALUE)
    rc, x_ref, st_ref = s.solve(eps=1e-10, maxit=100000)
    assert rc == 0
    rc, x_tight, _ = s.solve(eps=1e-14, maxit=100000)
    assert rc == 0
    g = Solver()
    g.load_model(m)
    g.build_pattern()
    # refused without the option, in both precisions
    g.assemble(_abi.FP64)
    rc, _ = g.solve(opts(mode=_abi.MODE_FP64, stop_rule=_abi.STOP_REF, tol=1e-10), raise_on_error=False)
    assert rc == _abi.ERR_ZERODIAG
    g.assemble(_abi.FP32)
    rc, _ = g.solve(opts(mode=_abi.MODE_MPIR, tol=1e-12), raise_on_error=False)
    assert rc == _abi.ERR_ZERODIAG
    # replaced with it: the reference's iteration count and solution
    g.set_zero_diagonal(VALUE)
    g.assemble(_abi.FP64)
    rc, st = g.solve(opts(mode=_abi.MODE_FP64, stop_rule=_abi.STOP_REF, tol=1e-10))
    assert rc == _abi.OK
    u = g.download()
    assert abs(st.iterations - st_ref.iterations) <= max(1, 0.02 * st_ref.iterations)
    assert np.linalg.norm(u - x_ref) <= 1e-8 * np.linalg.norm(x_ref)
    # the matrix keeps the replacement (SymmetricSparseMatrix after the solve)
    vals, _ = g.lower_values(_abi.FP64)
    rp, col, val = s.export_lower()
    dg, do = vals[rp[1:] - 1], val[rp[1:] - 1]
    bad = np.nonzero(np.abs(dg - do) > 1e-12 * np.abs(do))[0]
    assert len(bad) == 0, [(int(i), float(dg[i]), float(do[i]), int(m.restrained[i])) for i in bad[:8]]
    # mixed precision: FP32 matrix replaced, FP64 residual operator with the same entry
    g.assemble(_abi.FP32)
    rc, st = g.solve(opts(mode=_abi.MODE_MPIR, tol=1e-12))
    assert rc == _abi.OK
    u = g.download()
    assert np.linalg.norm(u - x_tight) <= 1e-8 * np.linalg.norm(x_tight)
    assert np.all(u[-m.ndpn:] == 0.0)  # nothing loads the unused node
