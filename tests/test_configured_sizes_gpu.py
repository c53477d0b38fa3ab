"""Parity at the configured sizes, through fe_solve on the GPU.

  * The LOBPCG configuration exactly: 24^3 7-point Dirichlet Laplacian + U[0,1)
    diagonal potential (n = 13,824), 8 lowest pairs, block 12, tol 1e-8, FP64.
    Checked against the oracle's restatement of the same loop on the same seeded
    input (eigenvalues within 1e-10 relative, iteration counts within 10 %) and
    against the dense spectrum (tests/golden/dense_spectra.json, LAPACK syevr):
    eigenvalues within 1e-10 relative. The reference's own LOBPCG (block = nev = 8,
    src/LOBPCGSolver.cpp:25-174) is checked the same way.
  * The generalized configuration's operator family at 20^3 (n = 8,000; 27-point
    stiffness with log-normal coefficients, M = M1 (x) M1 (x) M1): 64 lowest pairs by
    Jacobi-preconditioned LOBPCG and Davidson with a block of 96, FP64 against the
    oracle and the dense generalized spectrum, and precision=mixed against the dense
    spectrum.
Residuals are recomputed by the oracle from the returned vectors:
||K x - l M x|| / ((1 + |l|) ||M x||) <= tol.
"""
import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


def dense_lowest(key):
    return np.array(json.loads((GOLDEN / "dense_spectra.json").read_text())[key]["lowest"])


def solve(A, B=None, **kw):
    from fasteig_b200 import CsrMatrix, fasteig_options, fasteig_problem
    dA = CsrMatrix(A.rows, A.rowptr, A.colind, A.values)
    dB = CsrMatrix(B.rows, B.rowptr, B.colind, B.values) if B is not None else None
    opts = fasteig_options(A.rows)
    for k, v in kw.items():
        assert opts.set(k, v), k
    prob = fasteig_problem(dA, dB, solver=kw["solver"])
    prob.solve(opts)
    return prob


@pytest.fixture(scope="module")
def lobpcg24():
    from fasteig_b200 import matrices as M
    from oracle import oracle as O
    H = M.laplacian_uniform_potential(24, seed=0)
    return O.Csr(H.n, H.n, H.rowptr, H.colind, H.values)


@pytest.fixture(scope="module")
def km20():
    from fasteig_b200 import matrices as M
    from oracle import oracle as O
    K, Mm = M.stiffness_mass_27pt(20, seed=0)
    return (O.Csr(K.n, K.n, K.rowptr, K.colind, K.values),
            O.Csr(Mm.n, Mm.n, Mm.rowptr, Mm.colind, Mm.values))


def test_oracle_lobpcg_24cube_matches_dense(lobpcg24):
    """CPU: the oracle itself, at the configured size, against the dense spectrum."""
    from oracle import oracle as O
    ref = O.lobpcg_gen_solve(lobpcg24, 8, block=12, tol=1e-8, maxiter=1000, seed=1)
    np.testing.assert_allclose(ref.eigenvalues, dense_lowest("lobpcg_24cube_uniform_seed0")[:8],
                               rtol=1e-10, atol=0)


@pytest.mark.gpu
def test_lobpcg_24cube_block12_matches_oracle_and_dense(lobpcg24):
    from oracle import oracle as O
    ref = O.lobpcg_gen_solve(lobpcg24, 8, block=12, tol=1e-8, maxiter=1000, seed=1)
    p = solve(lobpcg24, solver="LOBPCG", nev=8, which="SR", tol=1e-8, maxiter=1000, seed=1,
              block=12)
    exp = dense_lowest("lobpcg_24cube_uniform_seed0")[:8]
    np.testing.assert_allclose(p.eigenvalues(), exp, rtol=1e-10, atol=0)
    np.testing.assert_allclose(p.eigenvalues(), ref.eigenvalues, rtol=1e-10, atol=0)
    assert abs(p.last_iterations() - ref.iterations) <= max(3, 0.1 * ref.iterations), \
        (p.last_iterations(), ref.iterations)
    assert np.all(p.residual_norms() <= 1.01e-8)
    final = O.residual_norms(lobpcg24, None, p.eigenvalues(), p.eigenvectors())
    assert np.all(final <= 1.01e-8), final


@pytest.mark.gpu
def test_lobpcg_24cube_reference_block_matches_oracle_and_dense(lobpcg24):
    """The reference's LOBPCG shape (block = nev = 8, no preconditioner)."""
    from oracle import oracle as O
    ref = O.lobpcg_solve(lobpcg24, 8, tol=1e-8, maxiter=2000, seed=1)
    p = solve(lobpcg24, solver="LOBPCG", nev=8, which="SR", tol=1e-8, maxiter=2000, seed=1)
    exp = dense_lowest("lobpcg_24cube_uniform_seed0")[:8]
    np.testing.assert_allclose(p.eigenvalues(), exp, rtol=1e-10, atol=0)
    np.testing.assert_allclose(p.eigenvalues(), ref.eigenvalues, rtol=1e-10, atol=0)
    assert abs(p.last_iterations() - ref.iterations) <= max(3, 0.1 * ref.iterations), \
        (p.last_iterations(), ref.iterations)
    final = O.residual_norms(lobpcg24, None, p.eigenvalues(), p.eigenvectors())
    assert np.all(final <= 1.01e-8), final


@pytest.mark.gpu
@pytest.mark.parametrize("solver", ["LOBPCG", "Davidson"])
def test_generalized_20cube_nev64_fp64_matches_oracle_and_dense(km20, solver):
    from oracle import oracle as O
    K, Mm = km20
    kw = dict(B=Mm, precond="jacobi", block=96, tol=1e-8, maxiter=3000, seed=1)
    if solver == "LOBPCG":
        ref = O.lobpcg_gen_solve(K, 64, **kw)
    else:
        ref = O.davidson_gen_solve(K, 64, maxblks=4, **kw)
    extra = {"maxblks": 4} if solver == "Davidson" else {}
    p = solve(K, Mm, solver=solver, nev=64, which="SR", tol=1e-8, maxiter=3000, seed=1,
              precond="jacobi", block=96, **extra)
    exp = dense_lowest("generalized_27pt_20cube_seed0")[:64]
    np.testing.assert_allclose(p.eigenvalues(), exp, rtol=1e-10, atol=1e-13)
    np.testing.assert_allclose(p.eigenvalues(), ref.eigenvalues, rtol=1e-10, atol=1e-13)
    assert abs(p.last_iterations() - ref.iterations) <= max(3, 0.1 * ref.iterations), \
        (p.last_iterations(), ref.iterations)
    final = O.residual_norms(K, Mm, p.eigenvalues(), p.eigenvectors())
    assert np.all(final <= 1.01e-8), final


@pytest.mark.gpu
@pytest.mark.parametrize("solver", ["LOBPCG", "Davidson"])
def test_generalized_20cube_nev64_mixed_against_dense(km20, solver):
    """precision=mixed (FP32 bulk, FP64 small steps, then FP64 to tol): the dense
    generalized spectrum to 1e-10 relative and oracle-recomputed residuals <= tol."""
    from oracle import oracle as O
    K, Mm = km20
    extra = {"maxblks": 4} if solver == "Davidson" else {}
    p = solve(K, Mm, solver=solver, nev=64, which="SR", tol=1e-8, maxiter=3000, seed=1,
              precond="jacobi", block=96, precision="mixed", **extra)
    exp = dense_lowest("generalized_27pt_20cube_seed0")[:64]
    np.testing.assert_allclose(p.eigenvalues(), exp, rtol=1e-10, atol=1e-13)
    final = O.residual_norms(K, Mm, p.eigenvalues(), p.eigenvectors())
    assert np.all(final <= 1.01e-8), final
    assert p.stats["fp32_iterations"] > 0, p.stats
