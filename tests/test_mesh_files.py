"""BETA mesh files (BasicMesh::ReadMesh / ReadMeshBinary): the reader follows
the reference layout -- header, optional processCommands block with the
coordinate read option, nodes numbered from 0 or 1, elements under their own
number -- and a model read from a file solves like the generated one."""
import numpy as np
import pytest

from betanoox_b200 import _abi, read_mesh, write_mesh
from betanoox_b200 import workloads as W


@pytest.mark.parametrize("binary", [False, True])
@pytest.mark.parametrize("first", [0, 1])
def test_round_trip(tmp_path, binary, first):
    for m in (W.cube_hex8(4), W.plate_quad4(5)):
        p = tmp_path / f"m{int(binary)}{first}"
        write_mesh(p, m.xyz, m.conn, binary=binary, first_number=first)
        xyz, conn = read_mesh(p, binary=binary)
        np.testing.assert_array_equal(conn, m.conn)
        np.testing.assert_array_equal(xyz, m.xyz)


def test_text_layout_with_commands_and_unsorted_elements(tmp_path):
    # a 2x1 quad4 strip in the y-z plane, read with setCoordinateReadOption yz,
    # nodes numbered from 1, elements listed out of order
    txt = """6 2 3
processCommands
setCoordinateReadOption yz
endCommands
1 0.0 0.0
2 1.0 0.0
3 2.0 0.0
4 0.0 1.0
5 1.0 1.0
6 2.0 1.0
2 4 2 3 6 5
1 4 1 2 5 4
"""
    p = tmp_path / "strip.msh"
    p.write_text(txt)
    xyz, conn = read_mesh(p)
    assert xyz.shape == (6, 3) and conn.shape == (2, 4)
    np.testing.assert_array_equal(xyz[:, 0], 0.0)  # x is not read with yz
    np.testing.assert_array_equal(xyz[1], [0.0, 1.0, 0.0])
    np.testing.assert_array_equal(conn, [[0, 1, 4, 3], [1, 2, 5, 4]])


def test_bad_files_are_rejected(tmp_path):
    p = tmp_path / "mixed.msh"
    p.write_text("4 2 2\n0 0 0\n1 1 0\n2 1 1\n3 0 1\n0 4 0 1 2 3\n1 3 0 1 2\n")
    with pytest.raises(_abi.BetaGpuError) as e:
        read_mesh(p)
    assert e.value.status == _abi.ERR_UNSUPPORTED
    q = tmp_path / "short.msh"
    q.write_text("4 1 2\n0 0 0\n1 1 0\n")
    with pytest.raises(_abi.BetaGpuError):
        read_mesh(q)
    r = tmp_path / "range.msh"
    r.write_text("3 1 2\n0 0 0\n1 1 0\n2 1 1\n0 4 0 1 2 7\n")
    with pytest.raises(_abi.BetaGpuError):
        read_mesh(r)


@pytest.mark.gpu
def test_a_model_read_from_a_mesh_file_solves(tmp_path, oracle):
    from betanoox_b200 import Solver, opts
    m = W.cube_hex8(6, seed=5)
    p = tmp_path / "cube.bin"
    write_mesh(p, m.xyz, m.conn, binary=True, first_number=1)
    xyz, conn = read_mesh(p, binary=True)
    mf = W.Model("from_file", m.kind, m.ndim, xyz, conn, m.ndpn, m.params, m.restrained, m.prescribed, m.load,
                 m.order)
    g = Solver()
    g.load_model(mf)
    g.build_pattern()
    g.assemble(_abi.FP32)
    g.solve(opts(tol=1e-12))
    u = g.download()
    s = oracle.System(m)
    s.set_bc(m.restrained, m.prescribed, m.load)
    s.build_pattern()
    s.assemble(m.params, m.order)
    _, ut, _ = s.solve(eps=1e-14, maxit=300000)
    assert np.linalg.norm(u - ut) / np.linalg.norm(ut) <= 1e-8
