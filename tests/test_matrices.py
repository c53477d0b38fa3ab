"""Synthetic benchmark-shape generators (host only)."""
import numpy as np
import pytest

from fasteig_b200 import matrices as M


def _sym_check(H):
    import scipy.sparse as sp
    A = sp.csr_matrix((H.values, H.colind, H.rowptr), shape=(H.n, H.n))
    assert abs(A - A.T).max() < 1e-15
    assert np.all(np.diff(H.rowptr) >= 1)
    for r in range(0, H.n, max(1, H.n // 50)):
        cols = H.colind[H.rowptr[r]:H.rowptr[r + 1]]
        assert np.all(np.diff(cols) > 0)


def test_laplacian_uniform_24cubed_nnz():
    H = M.laplacian_uniform_potential(24, 3, seed=0)
    assert H.n == 13824 and H.nnz == 93312
    _sym_check(H)
    diag = H.values[H.colind == np.repeat(np.arange(H.n), np.diff(H.rowptr))]
    assert np.all((diag >= 6.0) & (diag < 7.0))


@pytest.mark.parametrize("side", [8, 16])
def test_seven_point_wells_nnz_formula(side):
    H = M.laplacian_wells(side, wells=32, seed=3)
    assert H.nnz == side ** 3 + 6 * (side - 1) * side ** 2
    _sym_check(H)


def test_27pt_pair_nnz_and_definiteness():
    K, Mm = M.stiffness_mass_27pt(6, seed=1)
    assert K.nnz == Mm.nnz == (3 * 6 - 2) ** 3
    _sym_check(K)
    _sym_check(Mm)
    import scipy.sparse as sp
    Kd = sp.csr_matrix((K.values, K.colind, K.rowptr), shape=(K.n, K.n)).toarray()
    Md = sp.csr_matrix((Mm.values, Mm.colind, Mm.rowptr), shape=(Mm.n, Mm.n)).toarray()
    assert np.linalg.eigvalsh(Kd).min() > 0
    assert np.linalg.eigvalsh(Md).min() > 0
    m1 = np.diag(np.full(6, 2 / 3)) + np.diag(np.full(5, 1 / 6), 1) + np.diag(np.full(5, 1 / 6), -1)
    np.testing.assert_allclose(Md, np.kron(np.kron(m1, m1), m1), atol=1e-15)


def test_config2_nnz_formula_without_building():
    side = 128
    assert side ** 3 + 6 * (side - 1) * side ** 2 == 14581760
