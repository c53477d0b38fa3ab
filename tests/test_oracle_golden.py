"""Pin the CPU oracle against the reference's own known answers (no GPU).

* std::mt19937 + uniform_real_distribution(-1,1) (src/core/Executor.cpp:20-62)
  against the g++ build of oracle/rng_golden.cpp (tests/golden/mt19937.json).
* SiO.mtx, SR k=5, for Chebyshev, LOBPCG, Davidson, Krylov-Schur, Lanczos and block
  Lanczos against the
  ScaLAPACK spectrum tests/reference/SiO.out.121mpi, with the reference
  harness's rule |l - l_ref| <= 1e-10 + 1e-10 |l_ref| and residual <= 1e-8
  (tests/scripts/run_case.py:27-33,246-260; deck seed 1, tol 1e-8, maxiter 2000).
* Kuu/Muu generalized Krylov-Schur against tests/reference/KuuMuu_eig.txt.
"""
import json
import shutil
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT
from oracle import oracle as O

SR5 = dict(tol=1e-8, maxiter=2000, seed=1)


def test_mt19937_matches_libstdcxx_golden():
    gold = json.loads((GOLDEN / "mt19937.json").read_text())
    for seed, vals in gold.items():
        got = O.mt19937_uniform(len(vals), int(seed))
        np.testing.assert_array_equal(got, np.array(vals))


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_mt19937_matches_live_gxx_build(tmp_path):
    exe = tmp_path / "rng_golden"
    subprocess.run(["g++", "-O2", "-o", str(exe), str(ROOT / "oracle" / "rng_golden.cpp")], check=True)
    out = subprocess.run([str(exe), "3", "1000"], capture_output=True, text=True, check=True)
    np.testing.assert_array_equal(O.mt19937_uniform(1000, 3), np.array([float(x) for x in out.stdout.split()]))


def test_random_block_column_major_fill():
    B = O.random_block(7, 3, seed=5)
    flat = O.mt19937_uniform(21, 5)
    np.testing.assert_array_equal(B[:, 0], flat[:7])
    np.testing.assert_array_equal(B[:, 2], flat[14:])


def test_sio_fixture_shape(sio):
    assert sio.rows == 33401
    # 675,528 stored lower-triangle entries expand to 2*675528 - n_diag
    assert sio.nnz == 1317655
    A = sio.scipy()
    assert abs(A - A.T).max() == 0


def _check_sr5(res, spectra, A):
    exp = spectra["SiO"]["lowest"][:5]
    ok = O.eigenvalue_check(res.eigenvalues, exp)
    assert all(ok), (res.eigenvalues, exp)
    assert np.all(res.residual_norms <= 1e-8), res.residual_norms
    final = O.residual_norms(A, None, res.eigenvalues, res.eigenvectors)
    assert np.all(final <= 1.01e-8), final


@pytest.mark.parametrize("solver", ["chebyshev", "lobpcg", "davidson", "krylovschur",
                                    "lanczos", "blocklanczos"])
def test_sio_sr5_against_scalapack_spectrum(solver, sio, spectra):
    if solver == "chebyshev":
        res = O.chebyshev_solve(sio, 5, degree=10, **SR5)
    elif solver == "lobpcg":
        res = O.lobpcg_solve(sio, 5, **SR5)
    elif solver == "davidson":
        res = O.davidson_solve(sio, 5, **SR5)
    elif solver == "krylovschur":
        res = O.krylov_schur_solve(sio, 5, maxdim=40, **SR5)
    elif solver == "lanczos":
        # LanczosSolver: one chain, maxiter <= n (the deck's 2000 fits n = 33,401)
        res = O.lanczos_solve(sio, 5, **SR5)
    else:
        # BlockLanczosSolver with the deck's blksize 10
        res = O.block_lanczos_solve(sio, 5, 10, **SR5)
    _check_sr5(res, spectra, sio)


def test_sio_lr5_krylov_schur(sio, spectra):
    res = O.krylov_schur_solve(sio, 5, maxdim=40, which="lr", **SR5)
    exp = spectra["SiO"]["highest"][::-1][:5]
    assert all(O.eigenvalue_check(res.eigenvalues, exp)), (res.eigenvalues, exp)


def test_kuumuu_generalized_krylov_schur(kuumuu, spectra):
    K, M = kuumuu
    res = O.krylov_schur_solve(K, 5, maxdim=40, which="sm", B=M, **SR5)
    exp = spectra["KuuMuu"]["lowest"][:5]
    got = np.sort(res.eigenvalues)
    assert all(O.eigenvalue_check(got, exp, atol=1e-10, rtol=1e-9)), (got, exp)
    assert np.all(res.residual_norms <= 1e-8)


def test_spmm_restatement_matches_literal_loop():
    rng = np.random.default_rng(0)
    n = 40
    dense = rng.standard_normal((n, n)) * (rng.random((n, n)) < 0.2)
    dense = dense + dense.T
    r, c = np.nonzero(np.tril(dense))
    A = O.csr_from_triplets(n, r, c, dense[r, c], True)
    X = rng.standard_normal((n, 5))
    Y = rng.standard_normal((n, 5))
    lit = O.csr_spmm_reference_loop(A, X, 0.7, -0.3, Y)
    Y2 = Y.copy()
    O.csr_apply_block(A, X, 0, 5, Y2, 0.7, -0.3)
    np.testing.assert_allclose(Y2, lit, rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("which", ["sr", "lr"])
def test_chebyshev_hard_locking_extension_against_dense(which):
    """Hard-locking extension of the oracle's Chebyshev solver (QR and Rayleigh-Ritz
    on the active block only): eigenvalues equal the dense spectrum, true residuals
    reach tol, pairs come back in order."""
    from fasteig_b200 import matrices as M
    H = M.laplacian_wells(12, wells=8, seed=2)
    A = O.Csr(H.n, H.n, H.rowptr, H.colind, H.values)
    dense = np.linalg.eigvalsh(A.scipy().toarray())
    exp = dense[:24] if which == "sr" else dense[::-1][:24]
    res = O.chebyshev_solve(A, 24, degree=16, tol=1e-8, maxiter=300, seed=1, block=32,
                            bounds="ritz", amplification=1e6, locking="hard", which=which)
    np.testing.assert_allclose(res.eigenvalues, exp, rtol=1e-10, atol=1e-10)
    assert np.all(O.residual_norms(A, None, res.eigenvalues, res.eigenvectors) <= 1.01e-8)
    soft = O.chebyshev_solve(A, 24, degree=16, tol=1e-8, maxiter=300, seed=1, block=32,
                             bounds="ritz", amplification=1e6, which=which)
    assert res.iterations <= soft.iterations + 1


@pytest.mark.parametrize("which", ["lr", "sm", "lm", "be"])
def test_oracle_lanczos_selections_against_dense(which):
    """The oracle's LanczosSolver chain selects the reference's order (SR/LR/SM/LM/BE)
    and converges to the dense spectrum's pairs."""
    import scipy.sparse as sp
    from fasteig_b200 import matrices as M
    H = M.laplacian_uniform_potential(9, dim=3, seed=5)
    A = O.Csr(H.n, H.n, H.rowptr, H.colind, H.values)
    shifted = sp.csr_matrix(A.scipy() - 6.0 * sp.identity(H.n))  # spectrum on both sides of 0
    dense = shifted.toarray()
    S = O.Csr(H.n, H.n, shifted.indptr.astype(np.int32), shifted.indices.astype(np.int32),
              shifted.data)
    res = O.lanczos_solve(S, 4, tol=1e-9, maxiter=H.n, which=which, seed=2)
    w = np.linalg.eigvalsh(dense)
    order = {"lr": np.argsort(-w, kind="stable"), "sm": np.argsort(np.abs(w), kind="stable"),
             "lm": np.argsort(-np.abs(w), kind="stable"),
             "be": np.array([len(w) - 1, 0, len(w) - 2, 1])}[which]
    np.testing.assert_allclose(res.eigenvalues, w[order[:4]], rtol=1e-8, atol=1e-9)
    assert np.all(res.residual_norms <= 1e-9)


@pytest.mark.parametrize("solver", ["chebyshev", "lobpcg", "davidson", "krylovschur",
                                    "lanczos", "blocklanczos", "blockkrylovschur"])
def test_oracle_warm_start(solver):
    """fasteig_options::v0 semantics in the oracle: restarted from its own converged
    vectors a solver returns the same pairs in at most as many iterations; a v0 with the
    wrong row count is rejected as the reference rejects it."""
    from fasteig_b200 import matrices as M
    H = M.laplacian_wells(9, wells=4, seed=3)
    A = O.Csr(H.n, H.n, H.rowptr, H.colind, H.values)
    kw = dict(tol=1e-9, maxiter=400, seed=1)
    run = {"chebyshev": lambda **x: O.chebyshev_solve(A, 5, degree=8, **kw, **x),
           "lobpcg": lambda **x: O.lobpcg_solve(A, 5, **kw, **x),
           "davidson": lambda **x: O.davidson_solve(A, 5, **kw, **x),
           "krylovschur": lambda **x: O.krylov_schur_solve(A, 5, maxdim=30, **kw, **x),
           "lanczos": lambda **x: O.lanczos_solve(A, 5, **kw, **x),
           "blocklanczos": lambda **x: O.block_lanczos_solve(A, 5, 5, **kw, **x),
           "blockkrylovschur": lambda **x: O.block_krylov_schur_solve(A, 5, 5, maxdim=30, **kw,
                                                                     **x)}[solver]
    cold = run()
    warm = run(v0=cold.eigenvectors)
    np.testing.assert_allclose(warm.eigenvalues, cold.eigenvalues, rtol=1e-9, atol=1e-10)
    assert np.all(warm.residual_norms <= 1e-9)
    assert warm.iterations <= cold.iterations
    with pytest.raises(ValueError, match="v0"):
        run(v0=np.ones((H.n - 1, 5)))


def test_sio_lr5_block_lanczos(sio, spectra):
    res = O.block_lanczos_solve(sio, 5, 10, which="lr", **SR5)
    exp = spectra["SiO"]["highest"][::-1][:5]
    assert all(O.eigenvalue_check(res.eigenvalues, exp)), (res.eigenvalues, exp)
    assert np.all(res.residual_norms <= 1e-8)
