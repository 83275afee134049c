"""Row-sum form of the FP32 matrix (the batch engine's elasticity systems).

The batch kernel keeps each diagonal block as the block row sum S_I of the
FP64 operator and forms the product from differences,
    (A p)_I = sum_{J != I} A_IJ (p_J - p_I) + S_I p_I,
so that rounding the stored entries to FP32 leaves the rigid translations --
zero-energy modes away from the boundary -- exact.  These tests restate that
product in numpy on the oracle's assembled matrix (SymmetricSparseMatrix with
symmetric BC elimination) and check the property the kernel relies on, and
the iteration count it keeps on a long plate.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from betanoox_b200 import workloads as W


def _assembled(oracle, m):
    s = oracle.System(m)
    assert s.set_bc(m.restrained, m.prescribed, m.load) == 0
    s.build_pattern()
    assert s.assemble(m.params, m.order) == 0
    rp, col, val = s.export_lower()
    n = m.ndof
    rows = np.repeat(np.arange(n), np.diff(rp))
    L = sp.csr_matrix((val, (rows, col)), shape=(n, n))
    return (L + L.T - sp.diags(L.diagonal())).tocsr()


def _rowsum_product(A, nd, p):
    """FP32 row-sum form in FP64 arithmetic: off-diagonal blocks rounded to
    FP32, diagonal blocks replaced by the FP32-rounded FP64 block row sums."""
    c = A.tocoo()
    off = (c.row // nd) != (c.col // nd)
    v32 = c.data[off].astype(np.float32).astype(np.float64)
    r, k = c.row[off], c.col[off]
    self_idx = nd * (r // nd) + (k % nd)
    q = np.zeros(A.shape[0])
    np.add.at(q, r, v32 * (p[k] - p[self_idx]))
    S = np.zeros((A.shape[0], nd))
    np.add.at(S, (c.row, c.col % nd), c.data)
    S32 = S.astype(np.float32).astype(np.float64)
    base = nd * (np.arange(A.shape[0]) // nd)
    for j in range(nd):
        q += S32[:, j] * p[base + j]
    return q


@pytest.mark.parametrize("make", [lambda: W.plate_quad4(24), lambda: W.cube_hex8(6, seed=4)], ids=["quad4", "hex8"])
def test_translations_are_exact_in_the_rowsum_form(oracle, make):
    m = make()
    A = _assembled(oracle, m)
    nd = m.ndpn
    A32 = A.astype(np.float32).astype(np.float64)
    scale = abs(A).max()
    rest = np.asarray(m.restrained, dtype=bool)
    for j in range(nd):
        t = np.zeros(m.ndof)
        t[j::nd] = 1.0
        exact = A @ t  # block row sums of column j (unit rows on restrained dofs)
        rs = _rowsum_product(A, nd, t)
        plain = A32 @ t
        # every row within FP32 rounding of its own row sum
        assert np.abs(rs - exact)[~rest].max() <= 1e-6 * np.abs(exact).max() + 1e-12 * scale
        # interior rows (no restrained neighbour: the row sum vanishes): every
        # difference is zero and S_I is zero up to FP64 rounding, so the
        # row-sum form is exact there, while the plain FP32-rounded matrix
        # misses by ~eps32 * |A|
        inner = ~rest & (np.abs(exact) <= 1e-9 * scale)
        assert inner.sum() > 0.3 * m.ndof
        assert np.abs(rs - exact)[inner].max() <= 1e-9 * scale
        assert np.abs(plain - exact)[inner].max() >= 1e-8 * scale


def test_rowsum_form_is_the_matrix(oracle):
    """On a general vector the row-sum product equals A p to FP32 accuracy."""
    m = W.plate_quad4(16)
    A = _assembled(oracle, m)
    rng = np.random.default_rng(3)
    p = rng.standard_normal(m.ndof)
    p[np.asarray(m.restrained, dtype=bool)] = 0.0
    q = _rowsum_product(A, m.ndpn, p)
    ref = A @ p
    assert np.linalg.norm(q - ref) <= 1e-6 * np.linalg.norm(ref)


def _rowsum_matrix(A, nd):
    """The row-sum form as an explicit FP64 matrix: FP32-rounded off-diagonal
    blocks, diagonal blocks S_I - sum_{J != I} A32_IJ (S_I the FP64 block row
    sum rounded to FP32) -- the operator the batch kernel applies."""
    c = A.tocoo()
    diag = (c.row // nd) == (c.col // nd)
    v32 = c.data.astype(np.float32).astype(np.float64)
    od = sp.csr_matrix((np.where(diag, 0.0, v32), (c.row, c.col)), shape=A.shape)
    S = np.zeros((A.shape[0], nd))
    np.add.at(S, (c.row, c.col % nd), c.data)
    odsum = np.zeros((A.shape[0], nd))
    np.add.at(odsum, (c.row[~diag], c.col[~diag] % nd), v32[~diag])
    dv = S.astype(np.float32).astype(np.float64) - odsum
    rows = np.repeat(np.arange(A.shape[0]), nd)
    cols = ((nd * (np.arange(A.shape[0]) // nd))[:, None] + np.arange(nd)[None, :]).reshape(-1)
    return (od + sp.csr_matrix((dv.reshape(-1), (rows, cols)), shape=A.shape)).tocsr()


def _reliable_pcg(A, Aop, b, nd, tol=1e-10, delta=0.01, maxit=20000):
    """Block-Jacobi PCG in FP64 on the operator Aop with the residual replaced
    by the true b - A x whenever it has fallen by delta (the batch kernel's
    FP64-vector mode).  Returns the iterations to ||b - A x|| <= tol ||b||."""
    n = A.shape[0]
    nb = n // nd
    c = A.tocoo()
    m = (c.row // nd) == (c.col // nd)
    D = np.zeros((nb, nd, nd))
    D[c.row[m] // nd, c.row[m] % nd, c.col[m] % nd] = c.data[m]
    Minv = np.linalg.inv(D)
    prec = lambda r: np.einsum("bij,bj->bi", Minv, r.reshape(nb, nd)).reshape(-1)  # noqa: E731
    bn = np.linalg.norm(b)
    x, y, r = np.zeros(n), np.zeros(n), b.copy()
    z = prec(r)
    p, rho, maxrr = z.copy(), r @ z, r @ r
    for it in range(1, maxit + 1):
        q = Aop @ p
        a = rho / (p @ q)
        y += a * p
        r -= a * q
        z = prec(r)
        rz, rr = r @ z, r @ r
        maxrr = max(maxrr, rr)
        if rr < (0.5 * tol * bn) ** 2 or rr < delta * delta * maxrr:
            x += y
            y[:] = 0
            r = b - A @ x
            if np.linalg.norm(r) <= tol * bn:
                return it
            z = prec(r)
            rz = r @ z
            maxrr = r @ r
        p = z + (rz / rho) * p
        rho = rz
    return maxit


def test_rowsum_form_keeps_the_fp64_iteration_count(oracle):
    """The design claim behind the batch engine's precision: on a long plate
    from the serving mix, FP64 vectors on the plainly FP32-rounded matrix need
    a third more iterations than FP64, on the row-sum form almost none."""
    m = W.serve_request(99, 145)  # quad4 plate, 21,412 dofs
    A = _assembled(oracle, m)
    s = oracle.System(m)
    s.set_bc(m.restrained, m.prescribed, m.load)
    s.build_pattern()
    s.assemble(m.params, m.order)
    b = s.rhs()
    nd = m.ndpn
    it64 = _reliable_pcg(A, A, b, nd)
    it_plain = _reliable_pcg(A, A.astype(np.float32).astype(np.float64), b, nd)
    it_rs = _reliable_pcg(A, _rowsum_matrix(A, nd), b, nd)
    assert it_rs <= 1.05 * it64, (it64, it_rs)
    assert it_plain >= 1.2 * it64, (it64, it_plain)
