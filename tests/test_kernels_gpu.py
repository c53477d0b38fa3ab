"""Kernel parity on the GPU through the C ABI against the FP64 oracle.

Tolerances (componentwise, |.| applied entrywise):
  FP64 SpMM / Chebyshev step:  |Y - Y_ref| <= 1e-13 (|alpha| |A||X| + |gamma||X| + |beta||Z|)
  FP32 SpMM / Chebyshev step:  |Y - Y_ref| <= 4e-6  (same scale), FP32 accumulation
  Gram (FP64 accumulation):    |G - G_ref| <= 1e-13 |X|^T |Y|   (FP32 inputs: exact products)
  Rotation FP64:               |Y - Y_ref| <= 1e-13 |X||C|;  FP32: k * 2^-22 |X||C|
  Norms, Cholesky, inverse:    1e-12 relative
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def rand_sym_csr(n, density, seed, empty_rows=()):
    from oracle import oracle as O
    rng = np.random.default_rng(seed)
    nnz = max(1, int(density * n * n / 2))
    r = rng.integers(0, n, nnz)
    c = rng.integers(0, n, nnz)
    lo, hi = np.minimum(r, c), np.maximum(r, c)
    keep = ~np.isin(hi, empty_rows) & ~np.isin(lo, empty_rows)
    v = rng.standard_normal(nnz)
    diag = np.setdiff1d(np.arange(n), empty_rows)
    rows = np.concatenate([hi[keep], diag])
    cols = np.concatenate([lo[keep], diag])
    vals = np.concatenate([v[keep], rng.standard_normal(diag.size) + 4.0])
    return O.csr_from_triplets(n, rows, cols, vals, True)


def dev_csr(A):
    from fasteig_b200 import CsrMatrix
    return CsrMatrix(A.rows, A.rowptr, A.colind, A.values)


def block(n, b, dtype, seed, ld=None):
    g = torch.Generator().manual_seed(seed)
    ld = ld or b
    base = torch.randn(n, ld, generator=g, dtype=torch.float64)
    t = base.to(dtype).cuda()
    return t[:, :b] if ld != b else t


def absA(A):
    import scipy.sparse as sp
    return sp.csr_matrix((np.abs(A.values), A.colind, A.rowptr), shape=(A.rows, A.cols))


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("n,b", [(1, 1), (7, 3), (257, 1), (300, 2), (513, 5), (1000, 17),
                                 (777, 33), (600, 64), (400, 96), (1500, 320), (300, 1100)])
@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (-0.75, 1.0), (2.5, -0.5)])
def test_spmm_matches_oracle(dtype, n, b, alpha, beta):
    from fasteig_b200 import ops
    A = rand_sym_csr(n, min(0.05, 12.0 / n), seed=n + b, empty_rows=(0, n // 2) if n > 4 else ())
    dA = dev_csr(A)
    X = block(n, b, dtype, 1)
    Y = block(n, b, dtype, 2)
    if beta == 0.0:
        Y.fill_(float("nan"))  # beta == 0 must overwrite without reading
    X64 = X.double().cpu().numpy()
    Y64 = Y.double().cpu().numpy()
    ref = alpha * (A.scipy() @ X64) + (beta * Y64 if beta != 0.0 else 0.0)
    ops.spmm(dA, X, Y, alpha, beta)
    torch.cuda.synchronize()
    got = Y.double().cpu().numpy()
    scale = abs(alpha) * (absA(A) @ np.abs(X64)) + (abs(beta) * np.abs(Y64) if beta != 0 else 0.0)
    tol = 1e-13 if dtype == torch.float64 else 4e-6
    assert np.all(np.isfinite(got))
    assert np.all(np.abs(got - ref) <= tol * scale + 1e-300)


@pytest.fixture
def register_kernel():
    import fasteig_b200 as fe
    assert fe.lib.fe_set_spmm_kernel(1) == 0
    yield
    assert fe.lib.fe_set_spmm_kernel(0) == 0


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("stencil", ["star1", "star2", "box"])
@pytest.mark.parametrize("b", [16, 40, 320, 1000])
def test_pipelined_and_register_spmm_agree_on_stencils(dtype, stencil, b):
    """Every SpMM kernel (row-batched with 8- and 16-byte lanes, with and without
    the Z prefetch, loop, bulk-copy pipelined; 7/13/27-point rows) vs the oracle, including multi-panel and ragged
    panel widths and the fused Chebyshev epilogue."""
    import fasteig_b200 as fe
    from fasteig_b200 import matrices as M, ops
    from oracle import oracle as O
    if stencil == "box":
        H, _ = M.stiffness_mass_27pt(10, seed=1)
    else:
        H = M.laplacian_wells(10, wells=4, seed=1, stencil=stencil)
    A = O.Csr(H.n, H.n, H.rowptr, H.colind, H.values)
    dA = dev_csr(A)
    X = block(H.n, b, dtype, 1)
    Z = block(H.n, b, dtype, 2)
    Xn, Zn = X.double().cpu().numpy(), Z.double().cpu().numpy()
    ref = 0.7 * (A.scipy() @ Xn) - 0.2 * Xn - Zn
    outs = []
    for mode in (0, 1, 2, 3, 4, 5, 6, 7):
        assert fe.lib.fe_set_spmm_kernel(mode) == 0
        Zc = Z.clone()
        ops.cheb_step(dA, X, Zc, Zc, 0.7, -0.2, -1.0)
        torch.cuda.synchronize()
        outs.append(Zc.double().cpu().numpy())
    assert fe.lib.fe_set_spmm_kernel(0) == 0
    assert ops.device_status(clear=True) == 0
    scale = 0.7 * (absA(A) @ np.abs(Xn)) + 0.2 * np.abs(Xn) + np.abs(Zn)
    tol = 1e-13 if dtype == torch.float64 else 4e-6
    for got in outs:
        assert np.all(np.abs(got - ref) <= tol * scale + 1e-300)


def short_row_csr(n, max_nnz, seed):
    """Square CSR with 0..max_nnz random distinct columns per row (some rows
    empty, most without a stored diagonal)."""
    from oracle import oracle as O
    rng = np.random.default_rng(seed)
    rows, cols = [], []
    for r in range(n):
        k = int(rng.integers(0, max_nnz + 1))
        c = rng.choice(n, size=min(k, n), replace=False)
        rows.extend([r] * c.size)
        cols.extend(c.tolist())
    rows, cols = np.array(rows, dtype=np.int64), np.array(cols, dtype=np.int64)
    return O.csr_from_triplets(n, rows, cols, rng.standard_normal(rows.size), False)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("n,b", [(1, 16), (300, 16), (2000, 40), (5000, 320), (1200, 1000)])
@pytest.mark.parametrize("alpha,gamma,beta", [(1.0, 0.0, 0.0), (0.7, -0.2, -1.0), (-1.3, 0.4, 0.5)])
def test_pipelined_spmm_rows_without_diagonal(dtype, n, b, alpha, gamma, beta):
    """Bulk-copy pipelined kernel (mode 2) and the default kernel on rows of 0..7
    nonzeros, most without a stored diagonal (the gamma term then reads the row's
    own X row), some empty: oracle parity."""
    import fasteig_b200 as fe
    from fasteig_b200 import ops
    A = short_row_csr(n, 7, seed=n + b)
    dA = dev_csr(A)
    X = block(n, b, dtype, 1)
    Z = block(n, b, dtype, 2)
    Xn, Zn = X.double().cpu().numpy(), Z.double().cpu().numpy()
    ref = alpha * (A.scipy() @ Xn) + gamma * Xn + beta * Zn
    outs = []
    try:
        for mode in (2, 0, 4, 5, 6, 7):
            assert fe.lib.fe_set_spmm_kernel(mode) == 0
            Y = torch.full_like(X, float("nan"))
            ops.cheb_step(dA, X, Z, Y, alpha, gamma, beta)
            torch.cuda.synchronize()
            outs.append(Y.double().cpu().numpy())
    finally:
        assert fe.lib.fe_set_spmm_kernel(0) == 0
    assert ops.device_status(clear=True) == 0
    scale = abs(alpha) * (absA(A) @ np.abs(Xn)) + abs(gamma) * np.abs(Xn) + abs(beta) * np.abs(Zn)
    tol = 1e-13 if dtype == torch.float64 else 4e-6
    for got in outs:
        assert np.all(np.abs(got - ref) <= tol * scale + 1e-300)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_spmm_register_kernel_forced(dtype, register_kernel):
    from fasteig_b200 import ops
    n, b = 3000, 320
    A = rand_sym_csr(n, 0.003, seed=5)
    dA = dev_csr(A)
    X = block(n, b, dtype, 1)
    Y = block(n, b, dtype, 2)
    X64 = X.double().cpu().numpy()
    ops.spmm(dA, X, Y)
    torch.cuda.synchronize()
    tol = 1e-13 if dtype == torch.float64 else 4e-6
    assert np.all(np.abs(Y.double().cpu().numpy() - A.scipy() @ X64) <= tol * (absA(A) @ np.abs(X64)) + 1e-300)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_spmm_unaligned_leading_dimension_scalar_path(dtype):
    from fasteig_b200 import ops
    n, b = 333, 7
    A = rand_sym_csr(n, 0.03, seed=9)
    dA = dev_csr(A)
    Xs = block(n, b, dtype, 3, ld=11)  # ld not a multiple of the vector width
    Ys = block(n, b, dtype, 4, ld=13)
    X64 = Xs.double().cpu().numpy()
    ref = A.scipy() @ X64
    ops.spmm(dA, Xs, Ys)
    torch.cuda.synchronize()
    tol = 1e-13 if dtype == torch.float64 else 4e-6
    scale = absA(A) @ np.abs(X64)
    assert np.all(np.abs(Ys.double().cpu().numpy() - ref) <= tol * scale + 1e-300)


def test_spmm_rejects_overlapping_blocks():
    from fasteig_b200 import ops, FastEigError
    A = rand_sym_csr(50, 0.1, seed=1)
    dA = dev_csr(A)
    X = block(50, 8, torch.float64, 1)
    with pytest.raises(FastEigError):
        ops.spmm(dA, X, X)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("b", [1, 6, 40, 320])
def test_cheb_step_in_place_matches_oracle(dtype, b):
    from fasteig_b200 import ops
    n = 2000
    A = rand_sym_csr(n, 0.004, seed=b)
    dA = dev_csr(A)
    Ycur = block(n, b, dtype, 5)
    Yprev = block(n, b, dtype, 6)
    c, d = 0.31, -0.47
    Yc = Ycur.double().cpu().numpy()
    Yp = Yprev.double().cpu().numpy()
    ref = 2 * c * (A.scipy() @ Yc) + 2 * d * Yc - Yp
    ops.cheb_step(dA, Ycur, Yprev, Yprev, 2 * c, 2 * d, -1.0)  # in place over Y_{k-2}
    torch.cuda.synchronize()
    got = Yprev.double().cpu().numpy()
    scale = 2 * abs(c) * (absA(A) @ np.abs(Yc)) + 2 * abs(d) * np.abs(Yc) + np.abs(Yp)
    tol = 1e-13 if dtype == torch.float64 else 4e-6
    assert np.all(np.abs(got - ref) <= tol * scale + 1e-300)


@pytest.mark.parametrize("degree", [1, 2, 5, 16])
def test_cheb_filter_matches_oracle_recurrence(degree):
    from fasteig_b200 import ops
    from oracle import oracle as O
    n, b = 1200, 24
    A = rand_sym_csr(n, 0.005, seed=degree)
    dA = dev_csr(A)
    X = block(n, b, torch.float64, 7)
    S = torch.empty_like(X)
    X0 = X.cpu().numpy()
    lam = np.linalg.eigvalsh(A.scipy().toarray())
    lo, up = lam.min(), lam.max()
    c, d = O.chebyshev_filter_coefficients(lo, up, degree)
    ref = O.chebyshev_filter(lambda Z: A.scipy() @ Z, X0.copy(), degree, lo, up)
    ops.cheb_filter(dA, X, S, degree, c, d)
    torch.cuda.synchronize()
    got = X.cpu().numpy()
    np.testing.assert_allclose(got, ref, rtol=1e-11, atol=1e-11 * np.abs(ref).max())


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("n,k,m", [(1, 1, 1), (5, 3, 2), (1000, 17, 33), (20000, 64, 64),
                                   (70001, 130, 70), (4097, 320, 320)])
def test_gram_fp64_accumulation(dtype, n, k, m):
    from fasteig_b200 import ops
    X = block(n, k, dtype, 11)
    Y = block(n, m, dtype, 12)
    X64 = X.double().cpu().numpy()
    Y64 = Y.double().cpu().numpy()
    G = ops.gram(X, Y)
    torch.cuda.synchronize()
    ref = X64.T @ Y64
    scale = np.abs(X64).T @ np.abs(Y64)
    assert np.all(np.abs(G.cpu().numpy() - ref) <= 1e-13 * scale + 1e-300)


def test_gram_is_deterministic():
    from fasteig_b200 import ops
    X = block(50000, 48, torch.float32, 1)
    G1 = ops.gram(X, X).clone()
    G2 = ops.gram(X, X)
    assert torch.equal(G1, G2)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("n,k,m", [(1, 1, 1), (9, 4, 3), (1000, 17, 33), (5000, 320, 320),
                                   (3001, 130, 200)])
@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (-1.0, 1.0)])
def test_rotation_matches_oracle(dtype, n, k, m, alpha, beta):
    from fasteig_b200 import ops
    X = block(n, k, dtype, 21)
    Y = block(n, m, dtype, 22)
    Cm = torch.randn(k, m, dtype=torch.float64, generator=torch.Generator().manual_seed(5)).cuda()
    X64 = X.double().cpu().numpy()
    Y64 = Y.double().cpu().numpy()
    C64 = Cm.cpu().numpy()
    if dtype == torch.float32:
        C64 = C64.astype(np.float32).astype(np.float64)
    ref = alpha * X64 @ C64 + (beta * Y64 if beta else 0.0)
    ops.rotate(X, Cm, Y, alpha, beta)
    torch.cuda.synchronize()
    scale = np.abs(X64) @ np.abs(C64) + (np.abs(Y64) if beta else 0.0)
    tol = 1e-13 if dtype == torch.float64 else (k + 2) * 2.0 ** -22
    assert np.all(np.abs(Y.double().cpu().numpy() - ref) <= tol * scale + 1e-300)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("n,m", [(1, 1), (100, 7), (50000, 33), (3000, 320)])
def test_residual_norms(dtype, n, m):
    from fasteig_b200 import ops
    AX = block(n, m, dtype, 31)
    X = block(n, m, dtype, 32)
    lam = torch.linspace(-3, 2, m, dtype=torch.float64).cuda()
    R = torch.empty_like(X)
    rn, xn, rel = ops.residual_norms(AX, X, lam, R=R)
    torch.cuda.synchronize()
    A64 = AX.double().cpu().numpy()
    X64 = X.double().cpu().numpy()
    L = lam.cpu().numpy()
    Rref = A64 - X64 * L[None, :]
    tol = 1e-12 if dtype == torch.float64 else 1e-6
    np.testing.assert_allclose(rn.cpu().numpy(), np.linalg.norm(Rref, axis=0), rtol=tol)
    np.testing.assert_allclose(xn.cpu().numpy(), np.linalg.norm(X64, axis=0), rtol=1e-12)
    np.testing.assert_allclose(rel.cpu().numpy(), np.linalg.norm(Rref, axis=0) /
                               ((1 + np.abs(L)) * np.linalg.norm(X64, axis=0)), rtol=tol)
    np.testing.assert_allclose(R.double().cpu().numpy(), Rref, rtol=tol, atol=tol * np.abs(Rref).max())
    cn = ops.column_norms(X)
    np.testing.assert_allclose(cn.cpu().numpy(), np.linalg.norm(X64, axis=0), rtol=1e-12)


@pytest.mark.parametrize("k", [1, 2, 17, 33, 64, 100, 320, 500, 900])
def test_potrf_and_trinv(k):
    from fasteig_b200 import ops
    rng = np.random.default_rng(k)
    Z = rng.standard_normal((k + 5, k))
    G = Z.T @ Z + 0.1 * np.eye(k)
    R, info = ops.potrf_upper(torch.from_numpy(G).cuda())
    Rinv = ops.trinv_upper(R)
    torch.cuda.synchronize()
    assert int(info.item()) == 0
    Rn = R.cpu().numpy()
    np.testing.assert_allclose(Rn, np.linalg.cholesky(G).T, rtol=1e-10, atol=1e-12)
    assert np.all(np.tril(Rn, -1) == 0)
    np.testing.assert_allclose(Rn @ Rinv.cpu().numpy(), np.eye(k), atol=1e-10)


def test_potrf_reports_rank_loss_on_device():
    from fasteig_b200 import ops
    G = np.ones((4, 4))  # rank one: the second pivot vanishes
    _, info = ops.potrf_upper(torch.from_numpy(G).cuda())
    torch.cuda.synchronize()
    assert int(info.item()) == 2


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_autotuned_spmm_matches_oracle(dtype):
    """fe_csr_autotune records the fastest kernel for a block width; SpMMs of that
    width then use it and keep the componentwise bound."""
    from fasteig_b200 import matrices as M
    from fasteig_b200 import ops
    from oracle import oracle as O
    H = M.laplacian_wells(20, wells=4, seed=5)
    A = O.Csr(H.n, H.n, H.rowptr, H.colind, H.values)
    dA = dev_csr(A)
    mode = dA.autotune(96, "fp32" if dtype == torch.float32 else "fp64")
    assert mode in (0, 1, 2, 3)
    X = block(H.n, 96, dtype, 41)
    Y = torch.zeros_like(X)
    X64 = X.double().cpu().numpy()
    ops.spmm(dA, X, Y, -0.5, 0.0)
    torch.cuda.synchronize()
    ref = -0.5 * (A.scipy() @ X64)
    scale = 0.5 * (absA(A) @ np.abs(X64))
    tol = 1e-13 if dtype == torch.float64 else 4e-6
    assert np.all(np.abs(Y.double().cpu().numpy() - ref) <= tol * scale + 1e-300)


def test_batched_syevd_matches_numpy():
    """fe_syevd_batched_f64: eigenvalues within 1e-12 |A| of numpy's, eigenvectors
    orthonormal and satisfying A z = l z to 1e-12 |A|, for sizes 1..96 in one call."""
    from fasteig_b200 import ops
    sizes = [1, 2, 5, 17, 20, 33, 64, 95, 96]
    lda = 96
    rng = np.random.default_rng(3)
    A = np.zeros((len(sizes), lda, lda))
    for p, m in enumerate(sizes):
        B = rng.standard_normal((m, m))
        A[p, :m, :m] = B + B.T
    W, Z = ops.syevd_batched(torch.from_numpy(A).cuda(), sizes)
    W, Z = W.cpu().numpy(), Z.cpu().numpy()
    for p, m in enumerate(sizes):
        a = A[p, :m, :m]
        scale = np.abs(a).max() * m
        ref = np.linalg.eigvalsh(a)
        assert np.all(np.abs(W[p, :m] - ref) <= 1e-12 * scale), p
        z = Z[p, :m, :m]
        assert np.abs(z.T @ z - np.eye(m)).max() <= 1e-12 * m
        assert np.abs(a @ z - z * W[p, :m]).max() <= 1e-12 * scale


def test_block_diag_grouped_spmm():
    """An SpMM on fe_csr_block_diag(parts) equals each part's SpMM on its rows."""
    from fasteig_b200 import CsrMatrix, ops
    from oracle import oracle as O
    parts = [rand_sym_csr(n, 0.02, 10 + i) for i, n in enumerate([300, 1, 517, 64])]
    dev = [dev_csr(A) for A in parts]
    G = CsrMatrix.block_diag(dev)
    assert G.rows == sum(A.rows for A in parts) and G.nnz == sum(A.values.size for A in parts)
    X = block(G.rows, 40, torch.float64, 7)
    Y = torch.zeros_like(X)
    ops.spmm(G, X, Y, 1.0, 0.0)
    torch.cuda.synchronize()
    X64, Y64 = X.cpu().numpy(), Y.cpu().numpy()
    r0 = 0
    for A in parts:
        ref = A.scipy() @ X64[r0:r0 + A.rows]
        scale = absA(A) @ np.abs(X64[r0:r0 + A.rows])
        assert np.all(np.abs(Y64[r0:r0 + A.rows] - ref) <= 1e-13 * scale + 1e-300)
        r0 += A.rows
    G.close()


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("n,k", [(1, 1), (300, 20), (70001, 8), (5000, 9), (100003, 16), (777, 31), (40000, 32),
                                 (70001, 97), (2049, 128)])
def test_basis_times_vector_products(dtype, n, k):
    """Lanczos-shaped products (m = 1: V^T x and y = a V c + b y, the vector a
    strided column) keep the Gram and rotation bounds."""
    from fasteig_b200 import ops
    V = block(n, k, dtype, 51, ld=k + 3)
    Xw = block(n, 2, dtype, 52, ld=5)
    x = Xw[:, 1:2]
    V64, x64 = V.double().cpu().numpy(), x.double().cpu().numpy()
    G = ops.gram(V, x).cpu().numpy()
    ref = V64.T @ x64
    assert np.all(np.abs(G - ref) <= 1e-13 * (np.abs(V64).T @ np.abs(x64)) + 1e-300)
    c = torch.randn(k, 1, dtype=torch.float64, generator=torch.Generator().manual_seed(1)).cuda()
    c64 = c.cpu().numpy()
    if dtype == torch.float32:
        c64 = c64.astype(np.float32).astype(np.float64)
    y0 = x.double().cpu().numpy()
    ops.rotate(V, c, x, -1.0, 1.0)
    got = x.double().cpu().numpy()
    ref = y0 - V64 @ c64
    tol = 1e-13 if dtype == torch.float64 else (k + 2) * 2.0 ** -22
    assert np.all(np.abs(got - ref) <= tol * (np.abs(V64) @ np.abs(c64) + np.abs(y0)) + 1e-300)
