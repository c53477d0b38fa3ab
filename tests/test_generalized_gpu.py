"""Generalized (K u = l M u) and Jacobi-preconditioned LOBPCG / block Davidson on
the GPU through fe_solve (an extension: the reference's LOBPCGSolver and
DavidsonSolver are standard-only and unpreconditioned).

Pinned three ways:
  * against the CPU oracle's restatement of the same loops (oracle.lobpcg_gen_solve,
    oracle.davidson_gen_solve) on the same seeded inputs: eigenvalues within 1e-10
    relative, iteration counts within 3 (or 10 % on runs of hundreds of iterations);
  * against dense scipy.linalg.eigh(K, M): eigenvalues within 1e-10 relative;
  * against the reference's KuuMuu golden spectrum (tests/reference/KuuMuu_eig.txt,
    7,102 generalized eigenvalues) with the harness rule |dl| <= 1e-10 + 1e-10 |l|.
Residuals: ||K x - l M x|| / ((1 + |l|) ||M x||) <= tol, recomputed by the oracle.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def solve(A, B=None, **kw):
    from fasteig_b200 import CsrMatrix, fasteig_options, fasteig_problem
    dA = CsrMatrix(A.rows, A.rowptr, A.colind, A.values)
    dB = CsrMatrix(B.rows, B.rowptr, B.colind, B.values) if B is not None else None
    opts = fasteig_options(A.rows)
    for k, v in kw.items():
        assert opts.set(k, v), k
    prob = fasteig_problem(dA, dB, solver=kw.get("solver", "LOBPCG"))
    prob.solve(opts)
    return prob


@pytest.fixture(scope="module")
def km8():
    from fasteig_b200 import matrices as M
    from oracle import oracle as O
    K, Mm = M.stiffness_mass_27pt(8, seed=0)
    return (O.Csr(K.n, K.n, K.rowptr, K.colind, K.values),
            O.Csr(Mm.n, Mm.n, Mm.rowptr, Mm.colind, Mm.values))


@pytest.fixture(scope="module")
def dense_km8(km8):
    import scipy.linalg as sl
    K, Mm = km8
    return sl.eigh(K.scipy().toarray(), Mm.scipy().toarray(), eigvals_only=True)


@pytest.mark.parametrize("precond", ["none", "jacobi"])
def test_lobpcg_generalized_matches_oracle_and_dense(km8, dense_km8, precond):
    from oracle import oracle as O
    K, Mm = km8
    ref = O.lobpcg_gen_solve(K, 8, B=Mm, precond=precond, tol=1e-8, maxiter=500, seed=1)
    p = solve(K, Mm, solver="LOBPCG", nev=8, which="SR", tol=1e-8, maxiter=500, seed=1,
              precond=precond)
    np.testing.assert_allclose(p.eigenvalues(), ref.eigenvalues, rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(p.eigenvalues(), dense_km8[:8], rtol=1e-10, atol=1e-12)
    assert abs(p.last_iterations() - ref.iterations) <= max(3, 0.1 * ref.iterations), \
        (p.last_iterations(), ref.iterations)
    assert np.all(p.residual_norms() <= 1.01e-8)
    final = O.residual_norms(K, Mm, p.eigenvalues(), p.eigenvectors())
    assert np.all(final <= 1.01e-8), final


@pytest.mark.parametrize("precond", ["none", "jacobi"])
@pytest.mark.parametrize("which,nev,block", [("sr", 8, 8), ("sr", 13, 18), ("lr", 8, 12)])
def test_lobpcg_generalized_mixed_precision_against_dense(km8, dense_km8, precond, which, nev,
                                                          block):
    """precision=mixed: FP32 phase (FP32 SpMMs, split-TF32 Grams and rotations) to the
    FP32 floor, then FP64 iterations to tol from its Ritz vectors. Eigenvalues equal the
    dense generalized spectrum, residuals recomputed by the oracle reach tol, and both
    phases ran."""
    from oracle import oracle as O
    K, Mm = km8
    p = solve(K, Mm, solver="LOBPCG", nev=nev, which=which, tol=1e-8, maxiter=800, seed=1,
              precond=precond, block=block, precision="mixed")
    exp = dense_km8[:nev] if which == "sr" else dense_km8[::-1][:nev]
    np.testing.assert_allclose(p.eigenvalues(), exp, rtol=1e-10, atol=1e-12)
    assert np.all(p.residual_norms() <= 1.01e-8)
    final = O.residual_norms(K, Mm, p.eigenvalues(), p.eigenvectors())
    assert np.all(final <= 1.01e-8), final
    assert p.stats["fp32_iterations"] > 0 and p.stats["fp64_iterations"] > 0, p.stats


@pytest.mark.parametrize("precond", ["none", "jacobi"])
@pytest.mark.parametrize("which,nev,block", [("sr", 8, 8), ("lr", 7, 12)])
def test_davidson_generalized_mixed_precision_against_dense(km8, dense_km8, precond, which,
                                                            nev, block):
    """Davidson with precision=mixed: FP32 restarts to the FP32 floor, then FP64 to tol;
    dense generalized eigenvalues, oracle-recomputed residuals <= tol, both phases ran."""
    from oracle import oracle as O
    K, Mm = km8
    p = solve(K, Mm, solver="Davidson", nev=nev, which=which, tol=1e-8, maxiter=800, seed=1,
              precond=precond, block=block, maxblks=4, precision="mixed")
    exp = dense_km8[:nev] if which == "sr" else dense_km8[::-1][:nev]
    np.testing.assert_allclose(p.eigenvalues(), exp, rtol=1e-10, atol=1e-12)
    final = O.residual_norms(K, Mm, p.eigenvalues(), p.eigenvectors())
    assert np.all(final <= 1.01e-8), final
    assert p.stats["fp32_iterations"] > 0 and p.stats["fp64_iterations"] > 0, p.stats


def test_lobpcg_standard_mixed_precision_against_dense(wells_small):
    """precision=mixed on a standard problem (routed to the generalized loop with B = I)."""
    from oracle import oracle as O
    A, dense = wells_small
    p = solve(A, None, solver="LOBPCG", nev=10, which="SR", tol=1e-8, maxiter=800, seed=2,
              block=14, precision="mixed")
    np.testing.assert_allclose(p.eigenvalues(), dense[:10], rtol=1e-10, atol=1e-12)
    final = O.residual_norms(A, None, p.eigenvalues(), p.eigenvectors())
    assert np.all(final <= 1.01e-8), final


@pytest.mark.parametrize("precond", ["none", "jacobi"])
@pytest.mark.parametrize("which", ["sr", "lr"])
def test_davidson_generalized_matches_oracle_and_dense(km8, dense_km8, precond, which):
    from oracle import oracle as O
    K, Mm = km8
    ref = O.davidson_gen_solve(K, 8, B=Mm, precond=precond, tol=1e-8, maxiter=500, which=which,
                               seed=1, maxblks=4)
    p = solve(K, Mm, solver="Davidson", nev=8, which=which, tol=1e-8, maxiter=500, seed=1,
              precond=precond, maxblks=4)
    np.testing.assert_allclose(p.eigenvalues(), ref.eigenvalues, rtol=1e-10, atol=1e-12)
    exp = dense_km8[:8] if which == "sr" else dense_km8[::-1][:8]
    np.testing.assert_allclose(p.eigenvalues(), exp, rtol=1e-10, atol=1e-12)
    # Hundreds of iterations amplify last-bit differences of the reductions into
    # slightly different paths: iteration counts agree to 3 or 10 %.
    assert abs(p.last_iterations() - ref.iterations) <= max(3, 0.1 * ref.iterations), \
        (p.last_iterations(), ref.iterations)
    final = O.residual_norms(K, Mm, p.eigenvalues(), p.eigenvectors())
    assert np.all(final <= 1.01e-8), final


def test_lobpcg_block_larger_than_nev_standard(wells_small):
    """Standard problem, block 12 for 8 requested pairs (the 24^3 LOBPCG configuration's
    shape on a smaller grid), with and without Jacobi."""
    from oracle import oracle as O
    A, dense = wells_small
    for precond in ("none", "jacobi"):
        ref = O.lobpcg_gen_solve(A, 8, precond=precond, block=12, tol=1e-8, maxiter=500, seed=2)
        p = solve(A, solver="LOBPCG", nev=8, which="SR", tol=1e-8, maxiter=500, seed=2,
                  precond=precond, block=12)
        np.testing.assert_allclose(p.eigenvalues(), ref.eigenvalues, rtol=1e-10, atol=1e-12)
        np.testing.assert_allclose(p.eigenvalues(), dense[:8], rtol=1e-10, atol=1e-12)
        assert abs(p.last_iterations() - ref.iterations) <= max(3, 0.1 * ref.iterations)


@pytest.fixture(scope="module")
def wells_small():
    from fasteig_b200 import matrices as M
    from oracle import oracle as O
    H = M.laplacian_uniform_potential(10, seed=3)
    A = O.Csr(H.n, H.n, H.rowptr, H.colind, H.values)
    return A, np.linalg.eigvalsh(A.scipy().toarray())


@pytest.mark.parametrize("solver", ["LOBPCG", "Davidson"])
def test_generalized_kuumuu_known_answers(kuumuu, spectra, solver):
    from oracle import oracle as O
    K, Mm = kuumuu
    p = solve(K, Mm, solver=solver, nev=6, which="SR", tol=1e-8, maxiter=3000, seed=1,
              precond="jacobi", maxblks=6)
    exp = spectra["KuuMuu"]["lowest"][:6]
    assert all(O.eigenvalue_check(p.eigenvalues(), exp)), (p.eigenvalues(), exp)
    final = O.residual_norms(K, Mm, p.eigenvalues(), p.eigenvectors())
    assert np.all(final <= 1.01e-8), final


def test_generalized_rejects_shape_mismatch(km8):
    from fasteig_b200 import CsrMatrix, fasteig_options, fasteig_problem
    from fasteig_b200 import matrices as M
    K, _ = km8
    other = M.laplacian_uniform_potential(5, seed=0)
    dK = CsrMatrix(K.rows, K.rowptr, K.colind, K.values)
    dB = CsrMatrix(other.n, other.rowptr, other.colind, other.values)
    opts = fasteig_options(K.rows)
    opts.set("nev", 4)
    opts.set("solver", "LOBPCG")
    with pytest.raises(Exception, match="same shape"):
        fasteig_problem(dK, dB, solver="LOBPCG").solve(opts)


@pytest.mark.parametrize("generalized", [False, True])
def test_davidson_block_larger_than_nev(km8, wells_small, generalized):
    """Davidson on a block of 12 Ritz vectors for 8 requested pairs (Jacobi corrections),
    standard and generalized, against the oracle and dense eigh."""
    import scipy.linalg as sl
    from oracle import oracle as O
    if generalized:
        A, Bm = km8
        dense = sl.eigh(A.scipy().toarray(), Bm.scipy().toarray(), eigvals_only=True)
    else:
        (A, dense), Bm = wells_small, None
    ref = O.davidson_gen_solve(A, 8, B=Bm, precond="jacobi", block=12, tol=1e-8, maxiter=500,
                               seed=4, maxblks=4)
    p = solve(A, Bm, solver="Davidson", nev=8, which="SR", tol=1e-8, maxiter=500, seed=4,
              precond="jacobi", block=12, maxblks=4)
    np.testing.assert_allclose(p.eigenvalues(), ref.eigenvalues, rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(p.eigenvalues(), dense[:8], rtol=1e-10, atol=1e-12)
    assert abs(p.last_iterations() - ref.iterations) <= max(3, 0.1 * ref.iterations)
    final = O.residual_norms(A, Bm, p.eigenvalues(), p.eigenvectors())
    assert np.all(final <= 1.01e-8), final


@pytest.mark.parametrize("which", ["sr", "lr", "be"])
def test_krylov_schur_generalized_matches_oracle(km8, dense_km8, which):
    """B-metric Krylov-Schur on B^-1 A (the mass-matrix solve by device CG to 1e-14
    stands in for the reference's factorization) against the oracle, which applies B^-1
    with a sparse LU, and dense eigh(K, M)."""
    from oracle import oracle as O
    K, Mm = km8
    ref = O.krylov_schur_solve(K, 6, tol=1e-8, maxiter=300, which=which, seed=5, maxdim=24, B=Mm)
    p = solve(K, Mm, solver="KrylovSchur", nev=6, which=which, tol=1e-8, maxiter=300, seed=5,
              maxdim=24)
    np.testing.assert_allclose(p.eigenvalues(), ref.eigenvalues, rtol=1e-10, atol=1e-12)
    assert abs(p.last_iterations() - ref.iterations) <= 1, (p.last_iterations(), ref.iterations)
    assert p.status() == ref.status
    exp = O.select_reference(dense_km8, which, 6)
    # dense eigh carries ~1e-13 |K| absolute error of its own
    np.testing.assert_allclose(np.sort(p.eigenvalues()), np.sort(exp), rtol=1e-10, atol=1e-11)
    final = O.residual_norms(K, Mm, p.eigenvalues(), p.eigenvectors())
    np.testing.assert_allclose(p.residual_norms(), final, rtol=1e-6, atol=1e-15)


def test_krylov_schur_generalized_kuumuu_known_answers(kuumuu, spectra):
    from oracle import oracle as O
    K, Mm = kuumuu
    p = solve(K, Mm, solver="KrylovSchur", nev=5, which="SR", tol=1e-8, maxiter=2000, seed=1,
              maxdim=40)
    exp = spectra["KuuMuu"]["lowest"][:5]
    assert all(O.eigenvalue_check(p.eigenvalues(), exp)), (p.eigenvalues(), exp)
    assert p.status() == 0
    assert np.all(p.residual_norms() <= 1e-8), p.residual_norms()
