"""Solver parity on the GPU: the device-resident Chebyshev solver through
fe_solve against (a) the reference's known answers (SiO SR k=5, ScaLAPACK
spectrum, harness rule |dl| <= 1e-10 + 1e-10|l|, residual <= 1e-8) and (b) the
CPU oracle on the same seeded inputs (eigenvalues within 1e-10 relative,
residuals <= tol, eigenvectors by subspace angle)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def solve(A, **kw):
    from fasteig_b200 import CsrMatrix, fasteig_options, fasteig_problem
    dA = CsrMatrix(A.rows, A.rowptr, A.colind, A.values)
    opts = fasteig_options(A.rows)
    for k, v in kw.items():
        assert opts.set(k, v), k
    prob = fasteig_problem(dA, solver=kw.get("solver", "Chebyshev"))
    prob.solve(opts)
    return prob


def subspace_angle(X, Y):
    qx, _ = np.linalg.qr(X)
    qy, _ = np.linalg.qr(Y)
    s = np.linalg.svd(qx.T @ qy, compute_uv=False)
    return float(np.arccos(np.clip(s.min(), -1, 1)))


def test_chebyshev_sio_sr5_known_answers(sio, spectra):
    from oracle import oracle as O
    p = solve(sio, solver="Chebyshev", nev=5, which="SR", tol=1e-8, maxiter=2000, seed=1)
    exp = spectra["SiO"]["lowest"][:5]
    assert all(O.eigenvalue_check(p.eigenvalues(), exp)), (p.eigenvalues(), exp)
    assert np.all(p.residual_norms() <= 1e-8)
    final = O.residual_norms(sio, None, p.eigenvalues(), p.eigenvectors())
    assert np.all(final <= 1.01e-8), final


def test_chebyshev_matches_oracle_iteration_by_iteration(sio):
    from oracle import oracle as O
    ref = O.chebyshev_solve(sio, 5, degree=10, tol=1e-8, maxiter=2000, seed=1)
    p = solve(sio, solver="Chebyshev", nev=5, which="SR", tol=1e-8, maxiter=2000, seed=1)
    assert abs(p.last_iterations() - ref.iterations) <= 2, (p.last_iterations(), ref.iterations)
    np.testing.assert_allclose(p.eigenvalues(), ref.eigenvalues, rtol=1e-10, atol=1e-12)
    assert subspace_angle(p.eigenvectors(), ref.eigenvectors) < 1e-6


@pytest.fixture(scope="module")
def wells12():
    from fasteig_b200 import matrices as M
    from oracle import oracle as O
    H = M.laplacian_wells(12, wells=8, seed=2)
    return O.Csr(H.n, H.n, H.rowptr, H.colind, H.values)


@pytest.mark.parametrize("which", ["sr", "lr"])
def test_chebyshev_fp64_vs_oracle_reference_bounds(wells12, which):
    from oracle import oracle as O
    ref = O.chebyshev_solve(wells12, 6, degree=8, tol=1e-8, maxiter=400, which=which, seed=3)
    p = solve(wells12, solver="Chebyshev", nev=6, which=which, tol=1e-8, maxiter=400, seed=3,
              degree=8)
    np.testing.assert_allclose(p.eigenvalues(), ref.eigenvalues, rtol=1e-10, atol=1e-12)
    assert abs(p.last_iterations() - ref.iterations) <= 2
    dense = np.linalg.eigvalsh(wells12.scipy().toarray())
    exp = dense[:6] if which == "sr" else dense[::-1][:6]
    if ref.residual_norms.max() <= 1e-8:
        np.testing.assert_allclose(p.eigenvalues(), exp, rtol=1e-10, atol=1e-10)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_chebyshev_ritz_bounds_block_against_dense(wells12, precision):
    from oracle import oracle as O
    nev, blk = 24, 32
    p = solve(wells12, solver="Chebyshev", nev=nev, which="SR", tol=1e-8, maxiter=300, seed=1,
              degree=16, block=blk, bounds="ritz", precision=precision, amplification=1e6)
    dense = np.linalg.eigvalsh(wells12.scipy().toarray())
    assert np.all(p.residual_norms() <= 1e-8), p.residual_norms()
    np.testing.assert_allclose(p.eigenvalues(), dense[:nev], rtol=1e-10, atol=1e-10)
    final = O.residual_norms(wells12, None, p.eigenvalues(), p.eigenvectors())
    assert np.all(final <= 1.01e-8)
    if precision == "mixed":
        assert p.stats["fp32_iterations"] > 0


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("nev,blk,which", [(24, 32, "sr"), (23, 30, "sr"), (21, 27, "lr")])
def test_chebyshev_hard_locking_against_dense_and_oracle(wells12, precision, nev, blk, which):
    """locking=hard (QR and Rayleigh-Ritz on the active block only), aligned and
    unaligned active blocks: dense eigenvalues, FP64 residuals <= tol, ascending
    order, and (FP64) the oracle's hard-locking iteration count within 2."""
    from oracle import oracle as O
    kw = dict(degree=16, block=blk, bounds="ritz", amplification=1e6)
    p = solve(wells12, solver="Chebyshev", nev=nev, which=which, tol=1e-8, maxiter=300, seed=1,
              precision=precision, locking="hard", **kw)
    dense = np.linalg.eigvalsh(wells12.scipy().toarray())
    exp = dense[:nev] if which == "sr" else dense[::-1][:nev]
    assert np.all(p.residual_norms() <= 1e-8), p.residual_norms()
    np.testing.assert_allclose(p.eigenvalues(), exp, rtol=1e-10, atol=1e-10)
    final = O.residual_norms(wells12, None, p.eigenvalues(), p.eigenvectors())
    assert np.all(final <= 1.01e-8)
    if precision == "fp64":
        ref = O.chebyshev_solve(wells12, nev, tol=1e-8, maxiter=300, which=which, seed=1,
                                locking="hard", **kw)
        assert abs(p.last_iterations() - ref.iterations) <= 2, (p.last_iterations(),
                                                                 ref.iterations)


def test_chebyshev_ritz_bounds_matches_oracle(wells12):
    from oracle import oracle as O
    ref = O.chebyshev_solve(wells12, 12, degree=12, tol=1e-8, maxiter=300, seed=4, block=16,
                            bounds="ritz")
    p = solve(wells12, solver="Chebyshev", nev=12, which="SR", tol=1e-8, maxiter=300, seed=4,
              degree=12, block=16, bounds="ritz", amplification=1e300)
    np.testing.assert_allclose(p.eigenvalues(), ref.eigenvalues, rtol=1e-10, atol=1e-12)
    assert abs(p.last_iterations() - ref.iterations) <= 2


@pytest.mark.parametrize("solver", ["LOBPCG", "Davidson"])
def test_block_solvers_sio_sr5_known_answers(sio, spectra, solver):
    from oracle import oracle as O
    p = solve(sio, solver=solver, nev=5, which="SR", tol=1e-8, maxiter=2000, seed=1)
    exp = spectra["SiO"]["lowest"][:5]
    assert all(O.eigenvalue_check(p.eigenvalues(), exp)), (p.eigenvalues(), exp)
    assert np.all(p.residual_norms() <= 1.01e-8), p.residual_norms()
    final = O.residual_norms(sio, None, p.eigenvalues(), p.eigenvectors())
    assert np.all(final <= 1.01e-8), final


@pytest.mark.parametrize("which", ["sr", "lr"])
def test_lobpcg_matches_oracle(wells12, which):
    from oracle import oracle as O
    ref = O.lobpcg_solve(wells12, 6, tol=1e-8, maxiter=500, which=which, seed=2)
    p = solve(wells12, solver="LOBPCG", nev=6, which=which, tol=1e-8, maxiter=500, seed=2)
    np.testing.assert_allclose(p.eigenvalues(), ref.eigenvalues, rtol=1e-10, atol=1e-12)
    assert abs(p.last_iterations() - ref.iterations) <= 3, (p.last_iterations(), ref.iterations)
    assert subspace_angle(p.eigenvectors(), ref.eigenvectors) < 1e-6


@pytest.mark.parametrize("which", ["sr", "lr", "be", "lm"])
def test_davidson_matches_oracle(wells12, which):
    from oracle import oracle as O
    ref = O.davidson_solve(wells12, 6, tol=1e-8, maxiter=300, which=which, seed=3, maxblks=6)
    p = solve(wells12, solver="Davidson", nev=6, which=which, tol=1e-8, maxiter=300, seed=3,
              maxblks=6)
    np.testing.assert_allclose(p.eigenvalues(), ref.eigenvalues, rtol=1e-10, atol=1e-12)
    assert abs(p.last_iterations() - ref.iterations) <= 3, (p.last_iterations(), ref.iterations)
    assert np.all(p.residual_norms() <= 1.01e-8)


def test_krylov_schur_sio_sr5_known_answers(sio, spectra):
    from oracle import oracle as O
    p = solve(sio, solver="KrylovSchur", nev=5, which="SR", tol=1e-8, maxiter=2000, seed=1,
              maxdim=40)
    exp = spectra["SiO"]["lowest"][:5]
    assert all(O.eigenvalue_check(p.eigenvalues(), exp)), (p.eigenvalues(), exp)
    assert np.all(p.residual_norms() <= 1e-8), p.residual_norms()


@pytest.mark.parametrize("which", ["sr", "lr", "lm", "be"])
def test_krylov_schur_matches_oracle(wells12, which):
    from oracle import oracle as O
    ref = O.krylov_schur_solve(wells12, 6, tol=1e-8, maxiter=300, which=which, seed=5, maxdim=24)
    p = solve(wells12, solver="KrylovSchur", nev=6, which=which, tol=1e-8, maxiter=300, seed=5,
              maxdim=24)
    np.testing.assert_allclose(p.eigenvalues(), ref.eigenvalues, rtol=1e-10, atol=1e-12)
    assert abs(p.last_iterations() - ref.iterations) <= 1, (p.last_iterations(), ref.iterations)
