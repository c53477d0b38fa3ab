"""Block Krylov-Schur (BlockKrylovSchurSolver::solve, src/BlockKrylovSchurSolver.cpp:26-215).

CPU: the oracle's restatement reproduces the reference's own known answers (the SiO case
of tests/CMakeLists.txt:72-84 with the harness deck of tests/scripts/run_case.py:225-243:
SR, k = 5, blksize 10, maxdim 40, tol 1e-8, seed 1; ScaLAPACK spectrum, rule
|dl| <= 1e-10 + 1e-10 |l|).
GPU: the device solver through fe_solve against the same known answers and against the
oracle on the same seeded inputs (eigenvalues 1e-10 relative, restart counts within 10 %),
for SR and LR on a 3D well problem, with oracle-recomputed residuals <= tol.
"""
import numpy as np
import pytest

SIO_DECK = dict(nev=5, blksize=10, maxdim=40, tol=1e-8, maxiter=2000, seed=1)


def solve(A, **kw):
    from fasteig_b200 import CsrMatrix, fasteig_options, fasteig_problem
    dA = CsrMatrix(A.rows, A.rowptr, A.colind, A.values)
    opts = fasteig_options(A.rows)
    for k, v in kw.items():
        assert opts.set(k, v), k
    prob = fasteig_problem(dA, solver="BlockKrylovSchur")
    prob.solve(opts)
    return prob


def test_oracle_block_krylov_schur_sio_known_answers(sio, spectra):
    from oracle import oracle as O
    r = O.block_krylov_schur_solve(sio, which="sr", **SIO_DECK)
    assert r.status == 0
    assert all(O.eigenvalue_check(r.eigenvalues, spectra["SiO"]["lowest"][:5]))
    assert np.all(r.residual_norms <= 1e-8)


@pytest.mark.gpu
def test_block_krylov_schur_sio_known_answers_and_oracle(sio, spectra):
    from oracle import oracle as O
    ref = O.block_krylov_schur_solve(sio, which="sr", **SIO_DECK)
    p = solve(sio, solver="BlockKrylovSchur", which="SR", **SIO_DECK)
    assert p.status() == 0
    assert all(O.eigenvalue_check(p.eigenvalues(), spectra["SiO"]["lowest"][:5]))
    np.testing.assert_allclose(p.eigenvalues(), ref.eigenvalues, rtol=1e-10, atol=1e-12)
    assert abs(p.last_iterations() - ref.iterations) <= max(3, 0.1 * ref.iterations), \
        (p.last_iterations(), ref.iterations)
    final = O.residual_norms(sio, None, p.eigenvalues(), p.eigenvectors())
    assert np.all(final <= 1.01e-8), final


@pytest.mark.gpu
@pytest.mark.parametrize("which,nev,b,maxdim", [("sr", 6, 4, 24), ("lr", 5, 3, 0)])
def test_block_krylov_schur_matches_oracle(which, nev, b, maxdim):
    from fasteig_b200 import matrices as M
    from oracle import oracle as O
    H = M.laplacian_wells(10, wells=6, seed=4)
    A = O.Csr(H.n, H.n, H.rowptr, H.colind, H.values)
    kw = dict(nev=nev, blksize=b, maxdim=maxdim, tol=1e-8, maxiter=3000, seed=2)
    ref = O.block_krylov_schur_solve(A, which=which, **kw)
    p = solve(A, solver="BlockKrylovSchur", which=which.upper(), **kw)
    np.testing.assert_allclose(p.eigenvalues(), ref.eigenvalues, rtol=1e-10, atol=1e-12)
    assert abs(p.last_iterations() - ref.iterations) <= max(3, 0.1 * ref.iterations)
    final = O.residual_norms(A, None, p.eigenvalues(), p.eigenvectors())
    assert np.all(final <= 1.01e-8), final
