"""The threaded host operator that times the oracle at full size (oracle/cpu.py)
computes what the NumPy/SciPy parity path computes: filter steps and products to
1e-14 relative, and the same Chebyshev solve (eigenvalues to 1e-12 relative, the
same cycle count)."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def wells10():
    from fasteig_b200 import matrices as M
    from oracle import oracle as O
    H = M.laplacian_wells(10, wells=6, seed=1)
    return O.Csr(H.n, H.n, H.rowptr, H.colind, H.values)


@pytest.mark.parametrize("sign", [1.0, -1.0])
def test_threaded_filter_and_apply_match_numpy(wells10, sign):
    from oracle import cpu
    from oracle import oracle as O
    ref = O.NumpyChebyshevOps(wells10, sign)
    got = cpu.ThreadedChebyshevOps(wells10, sign, threads=3)
    X = np.random.default_rng(0).standard_normal((wells10.rows, 37))
    a, b = ref.apply(X), got.apply(X)
    assert np.abs(a - b).max() <= 1e-14 * np.abs(a).max()
    for deg in (1, 2, 7):
        fa = ref.filter_window(X.copy(), deg, 1.5, 12.5)
        fb = got.filter_window(X.copy(), deg, 1.5, 12.5)
        assert np.abs(fa - fb).max() <= 1e-13 * np.abs(fa).max(), deg
    fa = ref.filter(X.copy(), 6, -2.0, 12.5)
    fb = got.filter(X.copy(), 6, -2.0, 12.5)
    assert np.abs(fa - fb).max() <= 1e-13 * np.abs(fa).max()
    lam = np.linspace(-1, 3, 37)
    rn, xn = got.residual_norms(b, X, lam)
    np.testing.assert_allclose(rn, np.linalg.norm(b - X * lam[None, :], axis=0), rtol=1e-13)
    np.testing.assert_allclose(xn, np.linalg.norm(X, axis=0), rtol=1e-13)


@pytest.mark.parametrize("locking", ["soft", "hard"])
def test_threaded_chebyshev_solve_matches_numpy(wells10, locking):
    from oracle import cpu
    from oracle import oracle as O
    kw = dict(degree=12, tol=1e-8, maxiter=200, seed=2, block=16, bounds="ritz",
              amplification=1e6, locking=locking)
    ref = O.chebyshev_solve(wells10, 12, **kw)
    got = O.chebyshev_solve(wells10, 12, ops=cpu.ThreadedChebyshevOps(wells10, 1.0, threads=2), **kw)
    np.testing.assert_allclose(got.eigenvalues, ref.eigenvalues, rtol=1e-12, atol=1e-13)
    assert got.iterations == ref.iterations
    assert np.all(got.residual_norms <= 1e-8)


def test_cycles_generator_yields_every_cycle(wells10):
    from oracle import oracle as O
    progs = []
    for p in O.chebyshev_cycles(wells10, 8, degree=10, tol=1e-8, maxiter=200, seed=1, block=12,
                                locking="hard", bounds="ritz", amplification=1e6):
        progs.append((p.iteration, p.converged, p.result is not None))
    assert progs[-1][1] and progs[-1][2]
    assert [i for i, _, _ in progs] == list(range(1, len(progs) + 1))


@pytest.mark.parametrize("which", ["sr", "lr"])
def test_oracle_grouped_member_against_dense(which):
    """The oracle's restatement of one grouped Chebyshev member (whole-subspace filter,
    Cholesky QR twice, Rayleigh-Ritz) reaches tol with the dense spectrum's pairs."""
    from fasteig_b200 import matrices as M
    from oracle import oracle as O
    H = M.laplacian_wells(11, wells=6, seed=9, stencil="star2")
    A = O.Csr(H.n, H.n, H.rowptr, H.colind, H.values)
    r = O.grouped_chebyshev_member(A, 10, degree=10, tol=1e-8, maxiter=400, which=which,
                                   seed=3, bounds="ritz", amplification=1e6)
    w = np.linalg.eigvalsh(A.scipy().toarray())
    exp = w[:10] if which == "sr" else w[::-1][:10]
    assert r.status == 0
    np.testing.assert_allclose(r.eigenvalues, exp, rtol=1e-10, atol=1e-10)
    assert np.all(r.residual_norms <= 1e-8)
