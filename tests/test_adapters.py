"""BETA's interfaces over the C ABI (include/beta_gpu_adapters.hpp): a C++
program drives GPUAssembler / GPUPCGMatrix in the order BasicModel and
Equations call BasicAssembler / LargeMatrix, and its answers are checked
against the oracle.  Without a GPU the program builds and fails cleanly."""
import os
import struct
import subprocess

import numpy as np
import pytest

from betanoox_b200 import _abi
from betanoox_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "adapter_check.cpp")
LIBDIR = os.path.join(ROOT, "betanoox_b200", "_lib")


def _build(tmp_path):
    from betanoox_b200.build import build
    build()
    exe = os.path.join(str(tmp_path), "adapter_check")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
                    "-L", LIBDIR, "-lbeta_gpu", "-Wl,-rpath," + LIBDIR], check=True)
    return exe


def _write_model(path, m, precision, rule, tol, maxit=100000):
    p = np.ascontiguousarray(m.params, dtype=np.float64)
    with open(path, "wb") as f:
        f.write(struct.pack("12i", m.kind, m.ndim, m.nnode, m.nelem, m.nnpe, m.ndpn, m.order, p.shape[0],
                            p.shape[1], precision, rule, maxit))
        f.write(struct.pack("d", tol))
        for a, dt in ((m.xyz, np.float64), (m.conn, np.int32), (p, np.float64), (m.restrained, np.uint8),
                      (m.prescribed, np.float64), (m.load, np.float64)):
            f.write(np.ascontiguousarray(a, dtype=dt).tobytes())


def _read_out(path, n):
    raw = open(path, "rb").read()
    it = struct.unpack("i", raw[:4])[0]
    v = np.frombuffer(raw[4:], dtype=np.float64)
    return it, v[:n], v[n:2 * n], v[2 * n:3 * n], v[3 * n:4 * n]


def test_adapters_build_and_fail_cleanly_without_gpu(tmp_path):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("GPU present")
    except Exception:
        pass
    exe = _build(tmp_path)
    m = W.cube_hex8(3)
    model = os.path.join(str(tmp_path), "m.bin")
    _write_model(model, m, _abi.FP32, _abi.STOP_RB, 1e-10)
    r = subprocess.run([exe, model, os.path.join(str(tmp_path), "o.bin")], capture_output=True, text=True)
    assert r.returncode == 2 and "beta_gpu::Error" in r.stderr


CASES = {
    "rve_mixed": (lambda: W.rve_hex8(7, 4), _abi.FP32, _abi.STOP_RB, 1e-12),
    "plate_fp64_ref_rule": (lambda: W.plate_quad4(12), _abi.FP64, _abi.STOP_REF, 1e-10),
    "heat_steady_mixed": (lambda: W.serve_request(1, 6), _abi.FP32, _abi.STOP_RB, 1e-12),
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_adapters_follow_the_reference_call_sequence(tmp_path, oracle, name):
    make, precision, rule, tol = CASES[name]
    m = make()
    exe = _build(tmp_path)
    model, out = os.path.join(str(tmp_path), "m.bin"), os.path.join(str(tmp_path), "o.bin")
    _write_model(model, m, precision, rule, tol)
    r = subprocess.run([exe, model, out], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    it, x, y, diag, pseudo = _read_out(out, m.ndof)
    s = oracle.System(m)
    s.set_bc(m.restrained, m.prescribed, m.load)
    s.build_pattern()
    s.assemble(m.params, m.order)
    # the pseudo-load the reference's addMatrix accumulates
    assert np.abs(pseudo - s.pseudo_load()).max() <= 1e-12 * max(1.0, np.abs(s.pseudo_load()).max())
    _, ut, _ = s.solve(eps=1e-14, maxit=300000)
    assert it > 0
    assert np.linalg.norm(x - ut) / np.linalg.norm(ut) <= (1e-8 if rule == _abi.STOP_RB else 1e-6)
    # vectorProduct and operator() against the oracle's matrix
    y_ref = s.matvec(np.ones(m.ndof))
    scale = 1e-12 if precision == _abi.FP64 else 1e-5
    assert np.linalg.norm(y - y_ref) <= scale * 10 * np.linalg.norm(y_ref) + 1e-300
    rp, col, val = s.export_lower()
    d_ref = val[rp[1:] - 1]  # diagonal last in each row
    assert np.abs(diag - d_ref).max() <= scale * np.abs(d_ref).max()
