"""CPU checks of the oracle's generalized / Jacobi-preconditioned LOBPCG and block
Davidson restatements against dense scipy.linalg.eigh(K, M), before they are used
to pin the CUDA drivers."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def km6():
    import scipy.linalg as sl
    from fasteig_b200 import matrices as M
    from oracle import oracle as O
    K, Mm = M.stiffness_mass_27pt(6, seed=1)
    K = O.Csr(K.n, K.n, K.rowptr, K.colind, K.values)
    Mm = O.Csr(Mm.n, Mm.n, Mm.rowptr, Mm.colind, Mm.values)
    return K, Mm, sl.eigh(K.scipy().toarray(), Mm.scipy().toarray(), eigvals_only=True)


@pytest.mark.parametrize("precond", ["none", "jacobi"])
def test_oracle_lobpcg_generalized(km6, precond):
    from oracle import oracle as O
    K, Mm, dense = km6
    r = O.lobpcg_gen_solve(K, 6, B=Mm, precond=precond, tol=1e-9, maxiter=400, seed=1)
    np.testing.assert_allclose(r.eigenvalues, dense[:6], rtol=1e-10, atol=1e-12)
    assert np.all(O.residual_norms(K, Mm, r.eigenvalues, r.eigenvectors) <= 1.01e-9)
    # B-orthonormal Ritz vectors
    G = r.eigenvectors.T @ (Mm.scipy() @ r.eigenvectors)
    assert np.abs(G - np.eye(6)).max() < 1e-10


@pytest.mark.parametrize("which", ["sr", "lr", "be"])
def test_oracle_davidson_generalized(km6, which):
    from oracle import oracle as O
    K, Mm, dense = km6
    r = O.davidson_gen_solve(K, 6, B=Mm, precond="jacobi", tol=1e-9, maxiter=400, which=which,
                             seed=1, maxblks=4)
    if which == "sr":
        exp = dense[:6]
    elif which == "lr":
        exp = dense[::-1][:6]
    else:
        exp = np.array([dense[-1], dense[0], dense[-2], dense[1], dense[-3], dense[2]])
    np.testing.assert_allclose(np.sort(r.eigenvalues), np.sort(exp), rtol=1e-10, atol=1e-12)
    assert np.all(O.residual_norms(K, Mm, r.eigenvalues, r.eigenvectors) <= 1.01e-9)


def test_oracle_jacobi_preconditioner_speeds_up_and_block_option():
    from fasteig_b200 import matrices as M
    from oracle import oracle as O
    H = M.laplacian_uniform_potential(8, seed=0)
    A = O.Csr(H.n, H.n, H.rowptr, H.colind, H.values)
    dense = np.linalg.eigvalsh(A.scipy().toarray())
    r12 = O.lobpcg_gen_solve(A, 8, block=12, tol=1e-9, maxiter=400, seed=1)
    r8 = O.lobpcg_gen_solve(A, 8, tol=1e-9, maxiter=400, seed=1)
    np.testing.assert_allclose(r12.eigenvalues, dense[:8], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(r8.eigenvalues, dense[:8], rtol=1e-10, atol=1e-12)
    assert r12.iterations <= r8.iterations
