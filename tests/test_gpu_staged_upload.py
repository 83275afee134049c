"""Uploads of 4 MiB or more from pageable host memory go through the solver
context's pinned staging buffer in 32 MiB halves (a threaded host copy into
one half while the DMA of the other runs).  An 84^3 hex8 cube has a 72 MiB
slot map (three halves, the first one refilled after its copy), a 41 MiB
material array (two halves) and 14-18 MiB mesh and load arrays, so every
structure and mesh array of a build takes that path.  The operators
assembled from the staged structure must equal the FP64 matrix-free element
operator, which reads only the mesh, on the free dofs; and the same mesh,
material and boundary arrays passed in pinned memory (copied directly, not
staged) must give the same bits.
"""
import numpy as np
import pytest

from betanoox_b200 import Solver, _abi
from betanoox_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _pinned(a):
    import torch
    t = torch.empty(a.shape, dtype={np.float64: torch.float64, np.int32: torch.int32,
                                    np.uint8: torch.uint8}[a.dtype.type], pin_memory=True)
    t.numpy()[...] = a
    return t.numpy()


def test_staged_structure_and_mesh_uploads():
    m = W.cube_hex8(84, seed=4)
    assert m.nelem * m.nnpe * m.nnpe * 2 > 2 * (32 << 20)  # the slot map spans three halves
    free = m.restrained == 0
    u = np.random.default_rng(5).standard_normal(m.ndof)
    u[~free] = 0.0

    g = Solver()
    g.load_model(m)  # numpy arrays: pageable
    g.build_pattern()
    f = g.internal_force(u)
    g.assemble(_abi.FP64)
    y64 = g.matvec(u, _abi.FP64)
    g.assemble(_abi.FP32)
    y32 = g.matvec(u, _abi.FP32)
    nf = np.linalg.norm(f[free])
    assert np.linalg.norm(y64[free] - f[free]) <= 1e-12 * nf
    assert np.linalg.norm(y32[free] - f[free]) <= 1e-5 * nf

    pm = type(m)(m.name, m.kind, m.ndim, _pinned(m.xyz), _pinned(m.conn), m.ndpn, _pinned(m.params),
                 _pinned(m.restrained), _pinned(m.prescribed), _pinned(m.load), m.order, m.meta)
    h = Solver()
    h.load_model(pm)
    h.build_pattern()
    h.assemble(_abi.FP32)
    np.testing.assert_array_equal(h.matvec(u, _abi.FP32), y32)
