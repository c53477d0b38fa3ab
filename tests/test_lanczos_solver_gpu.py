"""LanczosSolver (the reference's default solver, src/LanczosSolver.cpp:29-163) on the
device through fe_solve: one scalar Lanczos chain with full reorthogonalization and
no restart, convergence checked every fifth step.

  * SiO SR k=5 against the ScaLAPACK spectrum (harness rule |dl| <= 1e-10 + 1e-10|l|,
    residual <= 1e-8), and against the oracle's chain on the same seeded start vector:
    the same stopping step and eigenvalues within 1e-10;
  * LR and BE selections and a generalized pair (B^-1 A through conjugate gradients)
    against dense spectra;
  * the reference's argument checks (maxiter >= nev, maxiter <= n).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def solve(A, B=None, want_vectors=True, **kw):
    from fasteig_b200 import CsrMatrix, fasteig_options, fasteig_problem
    dA = CsrMatrix(A.rows, A.rowptr, A.colind, A.values)
    dB = CsrMatrix(B.rows, B.rowptr, B.colind, B.values) if B is not None else None
    opts = fasteig_options(A.rows)
    for k, v in dict(dict(solver="Lanczos"), **kw).items():
        assert opts.set(k, v), k
    prob = fasteig_problem(dA, dB, solver="Lanczos")
    prob.solve(opts, want_vectors=want_vectors)
    return prob


def test_lanczos_sio_sr5(sio, spectra):
    from oracle import oracle as O
    p = solve(sio, nev=5, which="SR", tol=1e-8, maxiter=2000, seed=1)
    exp = spectra["SiO"]["lowest"][:5]
    assert all(O.eigenvalue_check(p.eigenvalues(), exp)), (p.eigenvalues(), exp)
    assert np.all(p.residual_norms() <= 1e-8)
    final = O.residual_norms(sio, None, p.eigenvalues(), p.eigenvectors())
    assert np.all(final <= 1.01e-8), final
    ref = O.lanczos_solve(sio, 5, tol=1e-8, maxiter=2000, seed=1)
    assert p.last_iterations() == ref.iterations, (p.last_iterations(), ref.iterations)
    np.testing.assert_allclose(p.eigenvalues(), ref.eigenvalues, rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("which", ["LR", "BE"])
def test_lanczos_selections_against_dense(which):
    from fasteig_b200 import matrices as M
    from oracle import oracle as O
    H = M.laplacian_uniform_potential(11, dim=3, seed=4)
    A = O.Csr(H.n, H.n, H.rowptr, H.colind, H.values)
    p = solve(A, nev=6, which=which, tol=1e-9, maxiter=600, seed=2)
    w = np.linalg.eigvalsh(A.scipy().toarray())
    exp = w[::-1][:6] if which == "LR" else np.array([w[-1], w[0], w[-2], w[1], w[-3], w[2]])
    np.testing.assert_allclose(p.eigenvalues(), exp, rtol=1e-8, atol=1e-9)
    assert np.all(p.residual_norms() <= 1e-9)


def test_lanczos_generalized_pair():
    from fasteig_b200 import matrices as M
    from oracle import oracle as O
    import scipy.linalg as sla
    K, Mm = M.stiffness_mass_27pt(8, seed=1)
    A = O.Csr(K.n, K.n, K.rowptr, K.colind, K.values)
    B = O.Csr(Mm.n, Mm.n, Mm.rowptr, Mm.colind, Mm.values)
    p = solve(A, B, nev=5, which="LM", tol=1e-8, maxiter=300, seed=1, want_vectors=False)
    w = sla.eigh(A.scipy().toarray(), B.scipy().toarray(), eigvals_only=True)
    exp = w[::-1][:5]
    np.testing.assert_allclose(np.sort(p.eigenvalues())[::-1], exp, rtol=1e-8)
    assert np.all(p.residual_norms() <= 1e-8)


def test_lanczos_argument_checks():
    from fasteig_b200 import FastEigError
    from fasteig_b200 import matrices as M
    from oracle import oracle as O
    H = M.laplacian_wells(6, wells=2, seed=1)
    A = O.Csr(H.n, H.n, H.rowptr, H.colind, H.values)
    with pytest.raises(FastEigError, match="maxiter must be >= nev"):
        solve(A, nev=10, maxiter=5)
    with pytest.raises(FastEigError, match="maxiter must be <= n"):
        solve(A, nev=4, maxiter=H.n + 1)
