"""Grouped Chebyshev engine (extension) on the GPU: standard problems of uneven
size advance together in grouped kernels over one concatenated block-diagonal
operator and leave as they converge.

  * every returned pair meets tol by the reference's relative residual, and the
    eigenvalues agree with dense numpy.linalg.eigh within the residual bound
    |lambda - theta| <= ||A x - theta x|| (x of unit norm);
  * a problem's result does not depend on the rest of its group: bit-identical
    alone and beside problems of the same stencil, equal to 1e-11 beside others;
  * which=LR, returned vectors, several groups (widths) in one batch, graph
    replays once the membership is stable, and an ineligible request's error.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def problem(side, stencil, seed):
    from fasteig_b200 import matrices as M
    return M.laplacian_wells(side, wells=6, seed=seed, stencil=stencil)


def opts(n, nev, tol=1e-8, which="SR", degree=10, seed=3, **extra):
    from fasteig_b200 import fasteig_options
    o = fasteig_options(n)
    kv = dict(solver="Chebyshev", nev=nev, which=which, tol=tol, maxiter=600, seed=seed,
              degree=degree, bounds="ritz", amplification=1e6)
    kv.update(extra)
    for k, v in kv.items():
        assert o.set(k, v), k
    return o


def dense(H):
    A = np.zeros((H.n, H.n))
    for i in range(H.n):
        A[i, H.colind[H.rowptr[i]:H.rowptr[i + 1]]] = H.values[H.rowptr[i]:H.rowptr[i + 1]]
    return A


def csr(H):
    from fasteig_b200 import CsrMatrix
    return CsrMatrix(H.n, H.rowptr, H.colind, H.values)


def test_grouped_pairs_against_dense():
    from fasteig_b200 import grouped_chebyshev
    specs = [(12, "star1", 8, 1), (11, "star2", 12, 2), (13, "star1", 20, 3),
             (10, "star2", 30, 4), (12, "star2", 6, 5)]
    Hs = [problem(s, st, sd) for s, st, _, sd in specs]
    mats = [csr(H) for H in Hs]
    o = [opts(H.n, nev) for H, (_, _, nev, _) in zip(Hs, specs)]
    out, batch = grouped_chebyshev(mats, o, want_vectors=True)
    assert batch["repacks"] >= 2  # members left at different cycles
    assert batch["graph_replays"] > 0
    for H, (_, _, nev, _), r in zip(Hs, specs, out):
        assert r["status"] == 0
        assert np.all(r["residual_norms"] <= 1e-8)
        lam = r["eigenvalues"]
        ref = np.linalg.eigvalsh(dense(H))[:nev]
        bound = 1e-8 * (1.0 + np.abs(lam)) * 1.01 + 1e-12
        assert np.all(np.abs(lam - ref) <= bound), np.max(np.abs(lam - ref) / bound)
        X = r["eigenvectors"]
        assert X.shape == (H.n, nev)
        A = dense(H)
        res = np.linalg.norm(A @ X - X * lam, axis=0) / ((1 + np.abs(lam)) *
                                                          np.linalg.norm(X, axis=0))
        assert np.all(res <= 1.5e-8)
        assert np.allclose(X.T @ X, np.eye(nev), atol=1e-10)
    widths = {r["width"] for r in out}
    assert widths == {32, 64}  # two groups ran side by side


def test_grouped_result_independent_of_group():
    from fasteig_b200 import grouped_chebyshev
    Hs = [problem(12, "star1", 21), problem(13, "star1", 22), problem(11, "star1", 23)]
    mats = [csr(H) for H in Hs]
    o = [opts(H.n, 10) for H in Hs]
    alone, _ = grouped_chebyshev(mats[:1], o[:1])
    together, _ = grouped_chebyshev(mats, o)
    assert np.array_equal(alone[0]["eigenvalues"], together[0]["eigenvalues"])
    assert np.array_equal(alone[0]["residual_norms"], together[0]["residual_norms"])
    assert alone[0]["iterations"] == together[0]["iterations"]
    # beside a 13-point operator (another SpMM kernel shape may be picked)
    H2 = problem(12, "star2", 24)
    mixed, _ = grouped_chebyshev([mats[0], csr(H2)], [o[0], opts(H2.n, 10)])
    np.testing.assert_allclose(mixed[0]["eigenvalues"], alone[0]["eigenvalues"], rtol=1e-11,
                               atol=1e-12)
    assert np.all(mixed[0]["residual_norms"] <= 1e-8)


def test_grouped_lr_and_single_path_agree():
    from fasteig_b200 import fasteig_problem, grouped_chebyshev
    H = problem(12, "star2", 31)
    A = csr(H)
    out, _ = grouped_chebyshev([A], [opts(H.n, 8, which="LR")])
    ref = np.sort(np.linalg.eigvalsh(dense(H)))[::-1][:8]
    lam = out[0]["eigenvalues"]
    assert np.all(out[0]["residual_norms"] <= 1e-8)
    np.testing.assert_allclose(np.sort(lam)[::-1], ref, rtol=1e-9)
    # the per-request FP64 Chebyshev path gives the same pairs (within tol)
    p = fasteig_problem(A, solver="Chebyshev")
    p.solve(opts(H.n, 8, which="LR"), want_vectors=False)
    np.testing.assert_allclose(np.sort(lam), np.sort(p.eigenvalues()), rtol=1e-9)


def test_grouped_rejects_ineligible():
    from fasteig_b200 import FastEigError, grouped_chebyshev
    H = problem(10, "star1", 41)
    with pytest.raises(FastEigError, match="not eligible"):
        grouped_chebyshev([csr(H)], [opts(H.n, 8, locking="hard")])


@pytest.mark.parametrize("k", [1, 7, 32, 64, 96, 128])
def test_chol_inv_batched(k):
    """fe_chol_inv_upper_batched_f64: R^{-1} of chol(G) for a batch (one CTA per
    matrix, shared memory) against numpy; a non-SPD member reports its pivot and
    leaves the others unaffected."""
    import torch
    import fasteig_b200 as fe
    rng = np.random.default_rng(k)
    count = 3
    Gs = []
    for p in range(count):
        M = rng.standard_normal((k, k))
        Gs.append(M @ M.T + k * np.eye(k))
    if k > 1:
        Gs[1] = Gs[1].copy()
        Gs[1][k // 2, k // 2] = -1.0  # not positive definite
        Gs[1][k // 2, :k // 2] = 0.0
        Gs[1][:k // 2, k // 2] = 0.0
    host = np.stack([g.T.copy() for g in Gs])  # column-major per matrix
    dG = torch.from_numpy(host).cuda()
    dR = torch.full((count, k, k), np.nan, dtype=torch.float64, device="cuda")
    info = torch.full((count,), -7, dtype=torch.int32, device="cuda")
    assert fe.lib.fe_chol_inv_upper_batched_f64(count, dG.data_ptr(), k, k, dR.data_ptr(), k,
                                                info.data_ptr(), None) == 0
    torch.cuda.synchronize()
    inf = info.cpu().numpy()
    for p in range(count):
        if k > 1 and p == 1:
            assert inf[p] >= 1
            continue
        assert inf[p] == 0
        Rinv = dR[p].cpu().numpy().T  # column-major -> matrix
        R = np.linalg.cholesky(Gs[p]).T
        ref = np.linalg.inv(R)
        assert np.allclose(np.tril(Rinv, -1), 0.0)
        assert np.abs(Rinv - ref).max() <= 1e-12 * np.abs(ref).max() * k


def test_grouped_mixed_precision():
    """precision=mixed members filter in FP32 in the FP32-filter group of their width,
    move to the FP64 group at their floor, and end with the FP64 path's pairs (tol
    1e-8 and 1e-6); alone and in a same-stencil group the results are bit-identical."""
    from fasteig_b200 import grouped_chebyshev
    specs = [(12, "star1", 8, 1e-8), (13, "star1", 12, 1e-8), (11, "star1", 10, 1e-6),
             (12, "star2", 20, 1e-8)]
    Hs = [problem(s, st, 60 + i) for i, (s, st, _, _) in enumerate(specs)]
    mats = [csr(H) for H in Hs]
    o = [opts(H.n, nev, tol=tol, precision="mixed") for H, (_, _, nev, tol) in zip(Hs, specs)]
    out, batch = grouped_chebyshev(mats, o)
    for H, (_, _, nev, tol), r in zip(Hs, specs, out):
        assert r["status"] == 0
        assert np.all(r["residual_norms"] <= tol)
        assert r["fp32_iterations"] >= 1
        lam = r["eigenvalues"]
        ref = np.linalg.eigvalsh(dense(H))[:nev]
        bound = tol * (1.0 + np.abs(lam)) * 1.01 + 1e-12
        assert np.all(np.abs(lam - ref) <= bound)
    assert any(r["iterations"] > r["fp32_iterations"] for r in out)  # some FP64 cycles ran
    alone, _ = grouped_chebyshev(mats[:1], o[:1])
    assert np.array_equal(alone[0]["eigenvalues"], out[0]["eigenvalues"])
    assert alone[0]["iterations"] == out[0]["iterations"]


def test_grouped_matches_oracle_member():
    """Each member against the oracle's restatement of the engine's per-member cycle
    (oracle.grouped_chebyshev_member: the reference's seeded start block, Lanczos bounds,
    filter, Cholesky QR twice, Rayleigh-Ritz, residuals): same cycle count, eigenvalues
    to 1e-9 relative."""
    from fasteig_b200 import grouped_chebyshev
    from oracle import oracle as O
    specs = [(12, "star1", 8, "SR"), (11, "star2", 12, "SR"), (12, "star2", 8, "LR")]
    Hs = [problem(s, st, 70 + i) for i, (s, st, _, _) in enumerate(specs)]
    out, _ = grouped_chebyshev([csr(H) for H in Hs],
                               [opts(H.n, nev, which=w) for H, (_, _, nev, w) in zip(Hs, specs)])
    for H, (_, _, nev, w), r in zip(Hs, specs, out):
        A = O.Csr(H.n, H.n, H.rowptr, H.colind, H.values)
        ref = O.grouped_chebyshev_member(A, nev, degree=10, tol=1e-8, maxiter=600,
                                         which=w.lower(), seed=3, bounds="ritz",
                                         amplification=1e6)
        assert abs(r["iterations"] - ref.iterations) <= 1, (r["iterations"], ref.iterations)
        np.testing.assert_allclose(r["eigenvalues"], ref.eigenvalues, rtol=1e-9, atol=1e-11)
        assert np.all(r["residual_norms"] <= 1e-8)
