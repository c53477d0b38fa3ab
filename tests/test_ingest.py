"""CSR ingestion: triplets -> full-storage CSR, as fasteig_problem::
build_sparse_matrix_from_triplets + build_csr_from_sparse_matrix
(src/fasteig_problem.cpp:474-607) build it with Eigen.

CPU: the oracle's restatement (duplicates summed left to right in input order,
symmetric / skew expansion, explicit zeros kept) on hand-made and random inputs.
GPU: fe_csr_create_from_triplets and fe_csr_create_from_matrix_market against the
oracle, bit for bit (rowptr, colind and the FP64 values), on the reference's own
fixtures (SiO, Kuu, Muu lower triangles) and on random inputs with duplicates."""
import numpy as np
import pytest


def test_oracle_sums_duplicates_in_input_order():
    from oracle import oracle as O
    r, c = np.array([0, 0, 0, 1]), np.array([1, 1, 1, 1])
    A = O.csr_from_triplets(2, r, c, np.array([1e16, 1.0, -1e16, 2.0]), False)
    assert A.values.tolist() == [0.0, 2.0]  # (1e16 + 1) - 1e16, left to right
    B = O.csr_from_triplets(2, r, c, np.array([1e16, -1e16, 1.0, 2.0]), False)
    assert B.values.tolist() == [1.0, 2.0]


def test_oracle_expansion_matches_dense_symmetrization():
    from oracle import oracle as O
    rng = np.random.default_rng(3)
    n = 40
    L = np.tril(rng.standard_normal((n, n)) * (rng.random((n, n)) < 0.2))
    r, c = np.nonzero(L)
    A = O.csr_from_triplets(n, r, c, L[r, c], True)
    np.testing.assert_array_equal(A.scipy().toarray(), L + L.T - np.diag(np.diag(L)))
    S = O.csr_from_triplets(n, r, c, L[r, c], False, expand_skew=True)
    np.testing.assert_array_equal(S.scipy().toarray(), L - L.T + np.diag(np.diag(L)))
    Z = O.csr_from_triplets(3, [0, 1], [0, 2], [0.0, 5.0], True)  # explicit zero kept
    assert Z.values.tolist() == [0.0, 5.0, 5.0] and Z.colind.tolist() == [0, 2, 1]


def test_oracle_rejects_bad_triplets():
    from oracle import oracle as O
    with pytest.raises(ValueError, match="out of bounds"):
        O.csr_from_triplets(3, [0, 3], [0, 0], [1.0, 1.0], True)
    with pytest.raises(ValueError, match="n <= 0"):
        O.csr_from_triplets(0, [], [], [], True)


def _same(dev, ref):
    rp, ci, va = dev.to_host()
    np.testing.assert_array_equal(rp, ref.rowptr)
    np.testing.assert_array_equal(ci, ref.colind)
    np.testing.assert_array_equal(va.view(np.uint64), ref.values.view(np.uint64))


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["SiO", "K", "M"])
def test_device_ingest_reference_fixtures_bit_exact(which):
    from pathlib import Path

    import fasteig_b200 as fe
    from oracle import oracle as O
    g = Path(__file__).resolve().parent / "golden"
    if which == "SiO":
        z = np.load(g / "SiO.npz")
        r, c, v = z["row"], z["col"], z["val"]
    else:
        z = np.load(g / "KuuMuu.npz")
        p = "k_" if which == "K" else "m_"
        r, c, v = z[p + "row"], z[p + "col"], z[p + "val"]
    n = int(z["n"])
    ref = O.csr_from_triplets(n, r, c, v, True)
    _same(fe.CsrMatrix.from_triplets(n, r, c, v, expand="symmetric"), ref)


@pytest.mark.gpu
@pytest.mark.parametrize("expand", ["none", "symmetric", "skew"])
def test_device_ingest_random_duplicates_bit_exact(expand):
    import fasteig_b200 as fe
    from oracle import oracle as O
    rng = np.random.default_rng({"none": 1, "symmetric": 2, "skew": 3}[expand])
    n, count = 5000, 60000
    r = rng.integers(0, n, count)
    c = rng.integers(0, n, count)
    if expand != "none":  # one triangle, as symmetric MatrixMarket files store it
        r, c = np.maximum(r, c), np.minimum(r, c)
    # heavy duplication with values whose sum depends on the order
    r = np.concatenate([r, r[:20000], r[:5000]])
    c = np.concatenate([c, c[:20000], c[:5000]])
    v = rng.standard_normal(r.size) * 10.0 ** rng.integers(-8, 9, r.size)
    v[::97] = 0.0
    ref = O.csr_from_triplets(n, r, c, v, expand == "symmetric", expand_skew=expand == "skew")
    _same(fe.CsrMatrix.from_triplets(n, r, c, v, expand=expand), ref)


@pytest.mark.gpu
def test_device_ingest_matrix_market_files(tmp_path):
    import fasteig_b200 as fe
    from oracle import oracle as O
    rng = np.random.default_rng(9)
    n = 300
    r = rng.integers(0, n, 2000)
    c = rng.integers(0, n, 2000)
    r, c = np.maximum(r, c), np.minimum(r, c)
    v = rng.standard_normal(r.size)
    for sym, exp_sym, exp_skew in (("symmetric", True, False), ("general", False, False),
                                   ("skew-symmetric", False, True)):
        path = tmp_path / f"{sym}.mtx"
        with open(path, "w") as f:
            f.write(f"%%MatrixMarket matrix coordinate real {sym}\n% comment\n{n} {n} {r.size}\n")
            for i, j, x in zip(r, c, v):
                f.write(f"{i + 1} {j + 1} {float(x)!r}\n")
        ref = O.csr_from_triplets(n, r, c, v, exp_sym, expand_skew=exp_skew)
        _same(fe.CsrMatrix.from_matrix_market(path), ref)
    path = tmp_path / "pattern.mtx"
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate pattern general\n{n} {n} {r.size}\n")
        for i, j in zip(r, c):
            f.write(f"{i + 1} {j + 1}\n")
    _same(fe.CsrMatrix.from_matrix_market(path), O.csr_from_triplets(n, r, c, np.ones(r.size), False))


@pytest.mark.gpu
def test_device_ingest_errors_and_solve(sio):
    from pathlib import Path

    import fasteig_b200 as fe
    from fasteig_b200 import fasteig_options, fasteig_problem
    with pytest.raises(fe.FastEigError, match="out of bounds"):
        fe.CsrMatrix.from_triplets(3, [0, 3], [0, 0], [1.0, 1.0], expand="symmetric")
    with pytest.raises(fe.FastEigError, match="n <= 0"):
        fe.CsrMatrix.from_triplets(0, [], [], [])
    g = Path(__file__).resolve().parent / "golden"
    z = np.load(g / "SiO.npz")
    dA = fe.CsrMatrix.from_triplets(int(z["n"]), z["row"], z["col"], z["val"], expand="symmetric")
    dB = fe.CsrMatrix(sio.rows, sio.rowptr, sio.colind, sio.values)
    out = []
    for A in (dA, dB):
        o = fasteig_options(sio.rows)
        for k, v in dict(solver="Chebyshev", nev=5, which="SR", tol=1e-8, maxiter=2000, seed=1).items():
            o.set(k, v)
        p = fasteig_problem(A, solver="Chebyshev")
        p.solve(o, want_vectors=False)
        out.append(p.eigenvalues().copy())
    np.testing.assert_array_equal(out[0], out[1])
