"""System exchange formats (sparse.cpp printMatrixAddressFormat[Upper],
printCompressedRowFormat; SparseMatrixUtility.cpp CSR ASCII/binary): the
layout of each file follows the reference writers, and every format reads
back what was written."""
import os

import numpy as np
import pytest

from betanoox_b200 import _abi, read_lower, write_lower
from betanoox_b200 import workloads as W

FORMATS = [_abi.FMT_ADDRESS_LOWER, _abi.FMT_ADDRESS_UPPER, _abi.FMT_COMPRESSED_ROW, _abi.FMT_CSR_ASCII,
           _abi.FMT_CSR_BINARY]

# 3x3 lower triangle [[4], [-1, 4.5], [0.1, 0, 2e-7]] without the zero
RP = np.array([0, 1, 3, 5])
COL = np.array([0, 0, 1, 0, 2])
VAL = np.array([4.0, -1.0, 4.5, 0.1, 2e-7])


def _w(v):
    """C++ default float output, width 24, 16 significant digits."""
    return f"{v:>24.16g}".replace("e-0", "e-0")


def test_address_lower_layout(tmp_path):
    p = tmp_path / "a.txt"
    write_lower(p, _abi.FMT_ADDRESS_LOWER, RP, COL, VAL)
    expect = ("1\n3 5\n"
              f"\t0 0 {_w(4.0)}\n"
              f"\t1 0 {_w(-1.0)}\t1 1 {_w(4.5)}\n"
              f"\t2 0 {_w(0.1)}\t2 2 {_w(2e-7)}\n")
    assert p.read_text() == expect


def test_address_upper_layout(tmp_path):
    p = tmp_path / "u.txt"
    write_lower(p, _abi.FMT_ADDRESS_UPPER, RP, COL, VAL)
    expect = ("2\n3 5\n"
              f"\t0 0 {_w(4.0)}\t0 1 {_w(-1.0)}\t0 2 {_w(0.1)}\n"
              f"\t1 1 {_w(4.5)}\n"
              f"\t2 2 {_w(2e-7)}\n")
    assert p.read_text() == expect


def test_compressed_row_layout(tmp_path):
    p = tmp_path / "c.txt"
    write_lower(p, _abi.FMT_COMPRESSED_ROW, RP, COL, VAL)
    expect = ("1-Lower triangular storage format\n3\n"
              f"1 {_w(4.0)} 0\n"
              f"2 {_w(-1.0)} 0 {_w(4.5)} 1\n"
              f"2 {_w(0.1)} 0 {_w(2e-7)} 2\n")
    assert p.read_text() == expect


def test_csr_layouts(tmp_path):
    p = tmp_path / "s.txt"
    write_lower(p, _abi.FMT_CSR_ASCII, RP, COL, VAL)
    lines = p.read_text().split("\n")
    assert lines[0] == "3 5"
    assert lines[1] == "0 1 3 5 "
    assert lines[2] == "0 0 1 0 2 "
    assert [float(x) for x in lines[3:8]] == list(VAL)
    assert lines[3] == f"{4.0:>24.16e}"
    b = tmp_path / "s.bin"
    write_lower(b, _abi.FMT_CSR_BINARY, RP, COL, VAL)
    raw = b.read_bytes()
    assert len(raw) == 8 + 4 * 4 + 4 * 5 + 8 * 5
    assert list(np.frombuffer(raw[:8], np.int32)) == [3, 5]
    assert list(np.frombuffer(raw[8:24], np.int32)) == [0, 1, 3, 5]


@pytest.mark.parametrize("fmt", FORMATS)
def test_round_trip_of_an_assembled_system(tmp_path, oracle, fmt):
    m = W.rve_hex8(5, 3)
    s = oracle.System(m)
    s.set_bc(m.restrained, m.prescribed, m.load)
    s.build_pattern()
    s.assemble(m.params, m.order)
    rp, col, val = s.export_lower()
    p = tmp_path / f"k{fmt}"
    write_lower(p, fmt, rp, col, val)
    rp2, col2, val2 = read_lower(p, fmt)
    np.testing.assert_array_equal(rp, rp2)
    np.testing.assert_array_equal(col, col2)
    if fmt == _abi.FMT_CSR_BINARY:
        np.testing.assert_array_equal(val, val2)
    else:  # 16 significant digits
        assert np.abs(val - val2).max() <= 1e-15 * np.abs(val).max()


def test_reader_rejects_a_wrong_format(tmp_path):
    p = tmp_path / "a.txt"
    write_lower(p, _abi.FMT_ADDRESS_LOWER, RP, COL, VAL)
    with pytest.raises(_abi.BetaGpuError):
        read_lower(p, _abi.FMT_ADDRESS_UPPER)
    with pytest.raises(_abi.BetaGpuError):
        read_lower(tmp_path / "missing", _abi.FMT_CSR_BINARY)


@pytest.mark.gpu
def test_export_of_the_gpu_matrix_matches_the_oracle(tmp_path, oracle):
    from betanoox_b200 import Solver
    m = W.cube_hex8(6, seed=3)
    s = oracle.System(m)
    s.set_bc(m.restrained, m.prescribed, m.load)
    s.build_pattern()
    s.assemble(m.params, m.order)
    rp, col, val = s.export_lower()
    g = Solver()
    g.load_model(m)
    g.build_pattern()
    g.assemble(_abi.FP64)
    p = tmp_path / "k.bin"
    g.export_matrix(p, _abi.FMT_CSR_BINARY)
    rp2, col2, val2 = read_lower(p, _abi.FMT_CSR_BINARY)
    np.testing.assert_array_equal(rp, rp2)
    np.testing.assert_array_equal(col, col2)
    assert np.abs(val - val2).max() <= 1e-12 * np.abs(val).max()
    q = tmp_path / "k.txt"
    g.export_matrix(q, _abi.FMT_ADDRESS_LOWER)
    assert q.read_text().startswith(f"1\n{m.ndof} {len(col)}\n")


def _sha(path):
    import hashlib
    with open(path, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()


_REF_FMT = {"address_lower": _abi.FMT_ADDRESS_LOWER, "address_upper": _abi.FMT_ADDRESS_UPPER,
            "compressed_row": _abi.FMT_COMPRESSED_ROW, "csr_ascii": _abi.FMT_CSR_ASCII,
            "csr_binary": _abi.FMT_CSR_BINARY}


@pytest.mark.parametrize("name", list(_REF_FMT))
def test_files_equal_the_reference_writers(tmp_path, oracle, name):
    """Byte for byte the files the reference's own writers produce (sparse.cpp,
    SparseMatrixUtility.cpp compiled unmodified): against their golden
    SHA-256, live where oracle/_ref is built, and read back by the
    reference's own CSR readers."""
    import json
    gold = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ref_exchange.json")))
    m = W.rve_hex8(5, 3)
    s = oracle.System(m)
    s.set_bc(m.restrained, m.prescribed, m.load)
    s.build_pattern()
    s.assemble(m.params, m.order)
    rp, col, val = s.export_lower()
    ours = tmp_path / "ours"
    write_lower(ours, _REF_FMT[name], rp, col, val)
    assert _sha(ours) == gold["sha256"][name]
    if oracle.RefLeaf.available():
        ref = oracle.RefLeaf()
        theirs = tmp_path / "theirs"
        if name.startswith("csr"):
            binary = name == "csr_binary"
            ref.write_csr(theirs, binary, rp, col, val)
            ia, ja, a = ref.read_csr(ours, binary)
            np.testing.assert_array_equal(ia, rp)
            np.testing.assert_array_equal(ja, col)
            assert np.abs(a - val).max() <= (0 if binary else 1e-15 * np.abs(val).max())
        else:
            ref.print_lower(theirs, {"address_lower": 1, "address_upper": 2, "compressed_row": 3}[name], rp, col, val)
        assert _sha(theirs) == _sha(ours)
