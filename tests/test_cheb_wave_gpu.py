"""Multi-step Chebyshev filter (cheb_wave_kernel: several filter steps per launch, each
step a level of warps trailing the previous one by the operator's bandwidth) against one
SpMM launch per step, through the C ABI.

The multi-step schedule changes only when each row is computed, not how: every row of
every step runs the single-step row kernel's arithmetic, so results must be equal bit
for bit (rtol = atol = 0) for both precisions, even and odd degrees, row counts that are
not a multiple of the 1024-row completion block, blocks narrower than a full panel, and
operators with a bandwidth of about n (each level waiting on nearly all of the previous
one, or, where the window does not fit L2, one step per launch). The filter recurrence
itself is checked against the oracle in
test_kernels_gpu.py::test_cheb_filter_matches_oracle_recurrence.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _filter(dA, X0, degree, c, d, wave):
    import fasteig_b200 as fe
    from fasteig_b200 import ops
    assert fe.lib.fe_set_cheb_wave_kernel(1 if wave else 0) == 0
    try:
        X = X0.clone()
        S = torch.empty_like(X)
        ops.cheb_filter(dA, X, S, degree, c, d)
        torch.cuda.synchronize()
    finally:
        fe.lib.fe_set_cheb_wave_kernel(0)
    import ctypes
    status = np.zeros(1, dtype=np.int32)
    assert fe.lib.fe_device_status(status.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), 1) == 0
    assert status[0] == 0, status
    return X


def _wells(side, wells=6, seed=0):
    from fasteig_b200 import CsrMatrix
    from fasteig_b200 import matrices as M
    H = M.laplacian_wells(side, wells=wells, seed=seed)
    return H, CsrMatrix(H.n, H.rowptr, H.colind, H.values)


@pytest.mark.parametrize("dtype,cols", [(torch.float32, 320), (torch.float32, 64),
                                        (torch.float32, 200), (torch.float64, 160),
                                        (torch.float64, 32)])
@pytest.mark.parametrize("degree", [16, 5, 2])
def test_wave_filter_bitwise_equal_to_single_steps(dtype, cols, degree):
    H, dA = _wells(40)  # 64,000 rows, bandwidth 1,600
    g = torch.Generator().manual_seed(cols + degree)
    X0 = torch.randn(H.n, cols, generator=g, dtype=torch.float64).to(dtype).cuda()
    # the spectrum of the wells operator lies in about [-4, 13]
    lo, hi = 1.0, 13.5
    c, d = 2.0 / (hi - lo), -(hi + lo) / (hi - lo)
    ref = _filter(dA, X0, degree, c, d, wave=False)
    out = _filter(dA, X0, degree, c, d, wave=True)
    assert torch.isfinite(ref).all()
    assert torch.equal(out, ref)


def test_wave_filter_ragged_rows_and_strided_block():
    """Rows not a multiple of the tile; a block with ld > ncols (the solver's views)."""
    from fasteig_b200 import CsrMatrix, ops
    import fasteig_b200 as fe
    from fasteig_b200 import matrices as M
    H = M.laplacian_wells(37, wells=4, seed=3)  # 50,653 rows
    dA = CsrMatrix(H.n, H.rowptr, H.colind, H.values)
    g = torch.Generator().manual_seed(7)
    base = torch.randn(H.n, 328, generator=g, dtype=torch.float64).float().cuda()
    outs = []
    for wave in (0, 1):
        assert fe.lib.fe_set_cheb_wave_kernel(wave) == 0
        X = base.clone()
        S = torch.zeros_like(X)
        Xv, Sv = X[:, :320], S[:, :320]
        assert fe.lib.fe_cheb_filter_f32(dA.handle, Xv.data_ptr(), Sv.data_ptr(), 328, 320, 9,
                                         0.15, -1.1, None) == 0
        torch.cuda.synchronize()
        outs.append(X)
    fe.lib.fe_set_cheb_wave_kernel(0)
    assert torch.equal(outs[0], outs[1])
    assert torch.equal(outs[1][:, 320:], base[:, 320:])  # columns past ncols untouched


def _permuted_path(n, seed):
    """1D Laplacian under a random symmetric permutation: 3 entries per row and a
    bandwidth of about n."""
    from oracle import oracle as O
    rng = np.random.default_rng(seed)
    perm = rng.permutation(n)
    i = np.arange(n - 1)
    rows = np.concatenate([perm[i + 1], perm])
    cols = np.concatenate([perm[i], perm])
    vals = np.concatenate([np.full(n - 1, -1.0), 2.0 + rng.random(n)])
    return O.csr_from_triplets(n, rows, cols, vals, True)


@pytest.mark.parametrize("n,cols", [(20000, 64), (300000, 320)])
def test_wave_filter_wide_bandwidth(n, cols):
    """Bandwidth ~ n: the small case runs the multi-step kernel with each level waiting
    on nearly all of the previous one (the block fits in L2); the large one has a
    window too large for L2 and runs one step per launch. Same results either way."""
    from fasteig_b200 import CsrMatrix
    A = _permuted_path(n, n)
    dA = CsrMatrix(A.rows, A.rowptr, A.colind, A.values)
    g = torch.Generator().manual_seed(n)
    X0 = torch.randn(n, cols, generator=g, dtype=torch.float64).float().cuda()
    ref = _filter(dA, X0, 6, 0.4, -1.2, wave=False)
    out = _filter(dA, X0, 6, 0.4, -1.2, wave=True)
    assert torch.isfinite(ref).all()
    assert torch.equal(out, ref)


def test_wave_filter_solver_bitwise_equal():
    """A mixed-precision Chebyshev solve gives the same result with and without it."""
    import fasteig_b200 as fe
    H, dA = _wells(32, wells=6, seed=2)
    res = []
    for wave in (0, 1):
        assert fe.lib.fe_set_cheb_wave_kernel(wave) == 0
        p = fe.fasteig_problem(dA, solver="Chebyshev")
        o = fe.fasteig_options()
        for k, v in dict(solver="Chebyshev", nev=24, which="SR", tol=1e-8, maxiter=300,
                         seed=1, degree=12, block=40, bounds="ritz", amplification=1e6,
                         precision="mixed", locking="hard").items():
            assert o.set(k, v), k
        p.solve(o, want_vectors=True)
        res.append((p.eigenvalues().copy(), p.stats["iterations"]))
    fe.lib.fe_set_cheb_wave_kernel(0)
    np.testing.assert_array_equal(res[0][0], res[1][0])
    assert res[0][1] == res[1][1]
