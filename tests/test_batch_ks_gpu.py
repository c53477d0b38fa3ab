"""Batched Krylov-Schur (extension) on the GPU: many standard problems solved in
lockstep by fe_batch_krylov_schur.

  * each problem against the CPU oracle's Krylov-Schur restatement
    (oracle.krylov_schur_solve, src/KrylovSchurSolver.cpp:28-160) on the same
    seeded start vector: eigenvalues within 1e-10 relative, restart counts within 1;
  * each problem alone (a batch of one) against the same problem inside the
    batch: bit-identical eigenvalues, residuals and iteration counts;
  * final relative residuals ||A y - l y|| / ((1 + |l|) ||y||) <= tol, recomputed
    by the oracle from the returned vectors.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def small_batch(count=12, seed=0):
    from fasteig_b200 import matrices as M
    rng = np.random.default_rng(seed)
    mats, nevs = [], []
    for i in range(count):
        side = int(rng.integers(9, 40))
        H = M.laplacian_uniform_potential(side, dim=2, seed=100 + i)
        mats.append(H)
        nevs.append(int(rng.choice([4, 8, 16])))
    return mats, nevs


def run_batch(mats, nevs, vectors=False, **kw):
    from fasteig_b200 import CsrMatrix, batch_krylov_schur, fasteig_options
    dev = [CsrMatrix(H.n, H.rowptr, H.colind, H.values) for H in mats]
    opts = fasteig_options()
    for k, v in dict(dict(which="SR", tol=1e-8, maxiter=300, seed=1), **kw).items():
        assert opts.set(k, v), k
    out, stats = batch_krylov_schur(dev, nevs, opts, want_vectors=vectors)
    return out, stats


@pytest.mark.parametrize("which", ["sr", "lr", "lm", "be"])
def test_batch_matches_oracle_per_problem(which):
    from oracle import oracle as O
    mats, nevs = small_batch(8, seed=1)
    out, stats = run_batch(mats, nevs, vectors=True, which=which)
    assert stats["rounds"] >= 1 and stats["graph_launches"] >= 20
    for H, nev, r in zip(mats, nevs, out):
        A = O.Csr(H.n, H.n, H.rowptr, H.colind, H.values)
        ref = O.krylov_schur_solve(A, nev, tol=1e-8, maxiter=300, which=which, seed=1)
        np.testing.assert_allclose(r["eigenvalues"], ref.eigenvalues, rtol=1e-10, atol=1e-12)
        assert abs(r["iterations"] - ref.iterations) <= 1, (r["iterations"], ref.iterations)
        final = O.residual_norms(A, None, r["eigenvalues"], r["eigenvectors"])
        np.testing.assert_allclose(r["residual_norms"], final, rtol=1e-6, atol=1e-15)
        if ref.residual_norms.max() <= 1e-8:
            assert np.all(final <= 1.01e-8)


def test_batch_result_same_alone_and_in_the_batch():
    mats, nevs = small_batch(10, seed=2)
    together, _ = run_batch(mats, nevs)
    for i in (0, 3, 9):
        alone, _ = run_batch([mats[i]], [nevs[i]])
        assert np.array_equal(alone[0]["eigenvalues"], together[i]["eigenvalues"])
        assert np.array_equal(alone[0]["residual_norms"], together[i]["residual_norms"])
        assert alone[0]["iterations"] == together[i]["iterations"]


def test_batch_known_dense_spectra_and_device_init():
    mats, nevs = small_batch(6, seed=3)
    out, _ = run_batch(mats, nevs, init="device")
    for H, nev, r in zip(mats, nevs, out):
        import scipy.sparse as sp
        dense = np.linalg.eigvalsh(
            sp.csr_matrix((H.values, H.colind, H.rowptr), shape=(H.n, H.n)).toarray())
        np.testing.assert_allclose(r["eigenvalues"], dense[:nev], rtol=1e-10, atol=1e-10)
        assert np.all(r["residual_norms"] <= 1e-8)


def test_batch_rejects_bad_input():
    from fasteig_b200 import CsrMatrix, FastEigError, batch_krylov_schur, fasteig_options
    from fasteig_b200 import matrices as M
    H = M.laplacian_uniform_potential(6, dim=2, seed=0)
    d = CsrMatrix(H.n, H.rowptr, H.colind, H.values)
    opts = fasteig_options()
    with pytest.raises(FastEigError):
        batch_krylov_schur([d], [H.n + 1], opts)
    H2 = M.laplacian_uniform_potential(20, dim=2, seed=0)
    d2 = CsrMatrix(H2.n, H2.rowptr, H2.colind, H2.values)
    opts.set("maxdim", 200)
    with pytest.raises(FastEigError, match="subspace dimension"):
        batch_krylov_schur([d2], [4], opts)
