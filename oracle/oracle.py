"""CPU oracle for the fasteig sparse symmetric eigensolver hot path.

TEST INFRASTRUCTURE ONLY. Nothing in the product path (``fasteig_b200``) may
import, call or link this module. It is imported by ``tests/``, by
``__graft_entry__.smoke()`` as the checker, and by ``bench.py``'s
``cpu_baseline`` leg / ``--impl reference`` arm, where it stands in for the
reference's CPU (Eigen) path, which cannot be compiled here because Eigen 3.4
is not installed (the reference fetches it over the network,
CMakeLists.txt:216,233-240).

It is a plain FP64 NumPy/SciPy restatement of the reference's CPU backend.
Every function names the reference file:line it follows (paths relative to
the fasteig project root). Third-party arithmetic used by the reference
(Eigen 3.4.0: ``SelfAdjointEigenSolver``, ``LLT``, ``HouseholderQR``,
``JacobiSVD``) is restated with the equivalent LAPACK routines through NumPy:
``eigh`` (syevd), ``cholesky`` (potrf), ``qr`` (geqrf/orgqr, same Householder
sign convention as Eigen's ``makeHouseholder``), ``svd`` (gesdd).

Parity pins (see tests/test_oracle_golden.py):
  * tests/reference/SiO.out.121mpi (33,401 ScaLAPACK eigenvalues of SiO.mtx):
    SR k=5 via Chebyshev, LOBPCG, Davidson and Krylov-Schur, checked with the
    reference harness's rule |dl| <= 1e-10 + 1e-10 |l_ref| and residual <= 1e-8
    (tests/scripts/run_case.py:246-260).
  * tests/reference/KuuMuu_eig.txt (7,102 generalized eigenvalues).
  * std::mt19937 / uniform_real_distribution bit-exact against a g++ build of
    oracle/rng_golden.cpp.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp

EPS = np.finfo(np.float64).eps

# --------------------------------------------------------------------------
# Random initial blocks: src/core/Executor.cpp:20-62
# std::mt19937(seed) + std::uniform_real_distribution<double>(-1, 1), with
# libstdc++'s generate_canonical<double, 53> drawing two 32-bit words per value
# (low word first). Column-major fill order.
# --------------------------------------------------------------------------


def mt19937_uniform(count: int, seed: int) -> np.ndarray:
    """``count`` draws of uniform_real_distribution<double>(-1,1) from mt19937(seed)."""
    bg = np.random.MT19937(0)
    bg._legacy_seeding(int(seed) & 0xFFFFFFFF)  # init_genrand(seed): std::mt19937(seed)
    raw = bg.random_raw(2 * count).astype(np.float64).reshape(count, 2)
    canon = (raw[:, 0] + raw[:, 1] * 4294967296.0) / 18446744073709551616.0
    canon = np.where(canon >= 1.0, np.nextafter(1.0, 0.0), canon)
    return 2.0 * canon - 1.0


def random_block(rows: int, cols: int, seed: int = 1) -> np.ndarray:
    """Executor::create_random_multivector (src/core/Executor.cpp:44-62)."""
    if rows <= 0 or cols <= 0:
        raise ValueError("Executor::create_random_multivector: dimensions must be positive.")
    # Column-major fill: column j takes draws [j*rows, (j+1)*rows) of one stream,
    # generated a column at a time (large blocks need no multi-GB temporaries).
    # (lo + hi * 2^32) is formed exactly as a 64-bit integer; its conversion to
    # double rounds once, as the double sum in generate_canonical does.
    bg = np.random.MT19937(0)
    bg._legacy_seeding(int(seed) & 0xFFFFFFFF)
    colmajor = np.empty((cols, rows))
    below_one = np.nextafter(1.0, 0.0)
    for j in range(cols):
        raw = bg.random_raw(2 * rows)
        canon = ((raw[1::2] << np.uint64(32)) | raw[0::2]).astype(np.float64)
        canon *= 1.0 / 18446744073709551616.0
        np.minimum(canon, below_one, out=canon)
        np.multiply(canon, 2.0, out=colmajor[j])
        colmajor[j] -= 1.0
    return np.ascontiguousarray(colmajor.T)


def random_vector(size: int, seed: int = 1) -> np.ndarray:
    """Executor::create_random_vector (src/core/Executor.cpp:20-34)."""
    if size <= 0:
        raise ValueError("Executor::create_random_vector: size must be positive.")
    return mt19937_uniform(size, seed)


def leading_block(v0: np.ndarray, n: int, b: int, solver: str) -> np.ndarray:
    """The block solvers' warm start: v0.leftCols(blksize), which must exist
    (src/BlockLanczosSolver.cpp:73-79, src/BlockKrylovSchurSolver.cpp:91-99)."""
    v0 = np.asarray(v0, dtype=np.float64)
    if v0.ndim == 1:
        v0 = v0[:, None]
    if v0.shape[0] != n or v0.shape[1] < b:
        raise ValueError(f"{solver}: v0 must have shape n x at least blksize.")
    return v0[:, :b].copy()


def warm_start(X: np.ndarray, v0: Optional[np.ndarray], max_cols: int, solver: str) -> np.ndarray:
    """The solvers' warm start over their seeded random block (fasteig_options::v0; e.g.
    src/ChebyshevSolver.cpp:96-103, src/LOBPCGSolver.cpp:49-56,
    src/DavidsonSolver.cpp:60-71): the first min(max_cols, v0 columns) columns of X are
    v0's."""
    if v0 is None:
        return X
    v0 = np.asarray(v0, dtype=np.float64)
    if v0.ndim == 1:
        v0 = v0[:, None]
    if v0.shape[0] != X.shape[0]:
        raise ValueError(f"{solver}: v0 row count does not match the problem.")
    k = min(max_cols, v0.shape[1])
    X = X.copy()
    X[:, :k] = v0[:, :k]
    return X


# --------------------------------------------------------------------------
# CSR matrices: include/core/CsrMatrix.hpp:18-27, src/core/CsrMatrix.cpp
# --------------------------------------------------------------------------


@dataclass
class Csr:
    rows: int
    cols: int
    rowptr: np.ndarray  # int32, rows+1
    colind: np.ndarray  # int32, nnz
    values: np.ndarray  # float64, nnz
    _sp: Optional[sp.csr_matrix] = field(default=None, repr=False)

    @property
    def nnz(self) -> int:
        return int(self.values.size)

    def scipy(self) -> sp.csr_matrix:
        if self._sp is None:
            self._sp = sp.csr_matrix((self.values, self.colind, self.rowptr),
                                     shape=(self.rows, self.cols))
        return self._sp


def validate_csr(A: Csr) -> None:
    """validate_csr_matrix_data (src/core/CsrMatrix.cpp:11-39)."""
    if A.rows < 0 or A.cols < 0:
        raise ValueError("CsrMatrixData: dimensions must be nonnegative.")
    if A.rowptr.size != A.rows + 1:
        raise ValueError("CsrMatrixData: rowptr size must be rows + 1.")
    if A.colind.size != A.values.size:
        raise ValueError("CsrMatrixData: colind and values sizes differ.")
    if A.rowptr.size and A.rowptr[0] != 0:
        raise ValueError("CsrMatrixData: rowptr must start at zero.")
    if A.rowptr.size and A.rowptr[-1] != A.values.size:
        raise ValueError("CsrMatrixData: rowptr end must equal nnz.")
    if np.any(np.diff(A.rowptr) < 0):
        raise ValueError("CsrMatrixData: rowptr must be nondecreasing.")
    if A.colind.size and (A.colind.min() < 0 or A.colind.max() >= A.cols):
        raise ValueError("CsrMatrixData: column index out of range.")


def csr_from_triplets(n: int, rows, cols, vals, expand_symmetric: bool,
                      expand_skew: bool = False) -> Csr:
    """Duplicate summation and symmetric expansion of triplets.

    fasteig_problem::build_sparse_matrix_from_triplets (src/fasteig_problem.cpp:474-506):
    Eigen's setFromTriplets sums duplicates left to right in input order. Then
    build_csr_from_sparse_matrix (src/fasteig_problem.cpp:554-607): every stored
    off-diagonal (r,c,v) of the merged matrix also contributes (c,r,v) (or -v when
    ``expand_skew``), positions holding two values keep their sum, rows are sorted by
    column (Eigen row-major compressed storage), explicit zeros are kept.
    """
    rows = np.asarray(rows, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    vals = np.asarray(vals, dtype=np.float64)
    if n <= 0:
        raise ValueError("Invalid matrix dimension n <= 0.")
    if rows.size and (rows.min() < 0 or cols.min() < 0 or rows.max() >= n or cols.max() >= n):
        raise ValueError("Triplet index out of bounds.")

    def merge(r, c, v):
        key = r * n + c
        order = np.argsort(key, kind="stable")  # equal keys stay in input order
        key, v = key[order], v[order]
        if key.size == 0:
            return key // n, key % n, v
        starts = np.flatnonzero(np.r_[True, key[1:] != key[:-1]])
        lengths = np.diff(np.r_[starts, key.size])
        acc = v[starts].copy()
        for t in range(1, int(lengths.max())):  # left-to-right sums (collapseDuplicates)
            more = lengths > t
            acc[more] = acc[more] + v[starts[more] + t]
        uk = key[starts]
        return uk // n, uk % n, acc

    r1, c1, v1 = merge(rows, cols, vals)
    if expand_symmetric or expand_skew:
        off = r1 != c1
        sign = -1.0 if expand_skew else 1.0
        r1, c1, v1 = merge(np.concatenate([r1, c1[off]]), np.concatenate([c1, r1[off]]),
                           np.concatenate([v1, sign * v1[off]]))
    rowptr = np.zeros(n + 1, dtype=np.int64)
    np.add.at(rowptr, r1 + 1, 1)
    rowptr = np.cumsum(rowptr)
    return Csr(n, n, rowptr.astype(np.int32), c1.astype(np.int32), v1.astype(np.float64))


def read_mtx(path) -> Csr:
    """MatrixMarket coordinate real {general,symmetric} reader (src/mmio.cpp:96 banner;
    1-based indices; symmetric files store one triangle and are expanded as in
    src/fasteig_problem.cpp:579-596)."""
    with open(path, "r") as f:
        banner = f.readline().lower().split()
        if len(banner) < 5 or banner[0] != "%%matrixmarket" or banner[2] != "coordinate":
            raise ValueError(f"{path}: unsupported MatrixMarket banner")
        symmetric = banner[4] == "symmetric"
        line = f.readline()
        while line.startswith("%"):
            line = f.readline()
        nr, nc, nz = (int(t) for t in line.split())
        data = np.loadtxt(f, dtype=np.float64, ndmin=2, max_rows=nz)
    if nr != nc:
        raise ValueError("CSR conversion requires a square matrix.")
    return csr_from_triplets(nr, data[:, 0].astype(np.int64) - 1,
                             data[:, 1].astype(np.int64) - 1, data[:, 2], symmetric)


def csr_apply_block(A: Csr, X: np.ndarray, first_col: int, block: int, Y: np.ndarray,
                    alpha: float = 1.0, beta: float = 0.0) -> None:
    """CpuCsrMatrix::apply_block (src/core/CsrMatrix.cpp:209-245):
    Y[:, :block] = beta*Y[:, :block] + alpha*A*X[:, first:first+block]; beta == 0
    overwrites (NaN-safe)."""
    if first_col < 0 or block <= 0 or first_col + block > X.shape[1]:
        raise ValueError("CpuCsrMatrix::apply_block: invalid column range.")
    if X.shape[0] != A.cols or Y.shape[0] != A.rows or Y.shape[1] < block:
        raise ValueError("CpuCsrMatrix::apply_block: dimension mismatch.")
    prod = A.scipy() @ X[:, first_col:first_col + block]
    if beta == 0.0:
        Y[:, :block] = alpha * prod
    else:
        Y[:, :block] = beta * Y[:, :block] + alpha * prod


def csr_spmm_reference_loop(A: Csr, X: np.ndarray, alpha: float, beta: float,
                            Y: np.ndarray) -> np.ndarray:
    """Literal row loop of src/core/CsrMatrix.cpp:227-244 (small cases only):
    scale Y by beta (or zero it), then for each nonzero in CSR order add
    (alpha*a) * X[col, :] to the row."""
    out = np.zeros_like(Y) if beta == 0.0 else beta * Y
    for r in range(A.rows):
        for k in range(A.rowptr[r], A.rowptr[r + 1]):
            out[r, :] += (alpha * A.values[k]) * X[A.colind[k], :]
    return out


# --------------------------------------------------------------------------
# QR factorizations: src/core/Orthogonalization.cpp
# --------------------------------------------------------------------------


def cholesky_qr(X: np.ndarray, gram: Optional[np.ndarray] = None):
    """cholesky_qr / cholesky_qr_from_gram (src/core/Orthogonalization.cpp:49-57,290-297).
    Returns (info, Q, R); info = -1 on rank loss (LLT failure)."""
    if gram is None:
        gram = X.T @ X
    try:
        L = np.linalg.cholesky(gram)
    except np.linalg.LinAlgError:
        return -1, None, None
    R = L.T
    # Q = X * R^{-1}, with R^{-1} from the triangular solve against the identity
    # (src/core/Orthogonalization.cpp:54-55).
    Rinv = sla.solve_triangular(R, np.eye(R.shape[0]), lower=False, check_finite=False)
    Q = X @ Rinv
    return 0, Q, R


def cholesky_qr2(X: np.ndarray):
    """cholesky_qr2 (src/core/Orthogonalization.cpp:299-315)."""
    info, q1, r1 = cholesky_qr(X)
    if info != 0:
        return info, None, None
    info, Q, r2 = cholesky_qr(q1)
    if info != 0:
        return info, None, None
    return 0, Q, r2 @ r1


def householder_qr(X: np.ndarray):
    """householder_qr (src/core/Orthogonalization.cpp:339-354): thin Q and upper R."""
    Q, R = np.linalg.qr(X, mode="reduced")
    return 0, Q, np.triu(R)


def weighted_cholesky_qr(X: np.ndarray, BX: np.ndarray):
    """B-weighted Cholesky QR (src/core/Orthogonalization.cpp:407-440): gram = X^T (BX),
    symmetrized before the factorization."""
    gram = X.T @ BX
    gram = 0.5 * (gram + gram.T)
    return cholesky_qr(X, gram)


def block_gram_schmidt(V: np.ndarray, k: int, S: np.ndarray, dual: Optional[np.ndarray] = None):
    """block_gram_schmidt (src/core/Orthogonalization.cpp:482-527): two-pass classical
    block GS of S against V[:, :k]. Returns (info, residual, H)."""
    if k == 0:
        return 0, S.copy(), np.zeros((0, S.shape[1]))
    Vk = V[:, :k]
    BV = (dual if dual is not None else V)[:, :k]
    H = BV.T @ S
    R = S - Vk @ H
    S2 = BV.T @ R
    H = H + S2
    R = R - Vk @ S2
    return 0, R, H


def orthonormalize_block(basis: np.ndarray, k: int, source: np.ndarray,
                         rank_tolerance: float = 1e-12) -> Optional[np.ndarray]:
    """orthonormalize_block (src/core/Orthogonalization.cpp:717-775)."""
    n = source.shape[0]
    if k == n:
        return None
    current = source
    result = None
    for _ in range(2):
        norms = np.linalg.norm(current, axis=0)
        if not np.all(np.isfinite(norms)):
            raise RuntimeError("orthonormalize_block: non-finite column norms.")
        scale = norms.max()
        if scale == 0.0:
            return None
        _, orth, _ = block_gram_schmidt(basis, k, current)
        _, Q, R = householder_qr(orth)
        U, s, _ = np.linalg.svd(R)
        capacity = min(current.shape[1], n - k)
        rank = 0
        while rank < capacity and s[rank] > rank_tolerance * scale:
            rank += 1
        if rank == 0:
            return None
        result = Q @ U[:, :rank]
        current = result
    return result


# --------------------------------------------------------------------------
# Ritz extraction: src/core/RitzExtraction.cpp, include/fasteig_solver.hpp:58-82
# --------------------------------------------------------------------------


def sort_indices(v: np.ndarray, which: str) -> np.ndarray:
    """sort_indices (include/fasteig_solver.hpp:58-82): stable sorts."""
    if which == "sr":
        return np.argsort(v, kind="stable")
    if which == "lr":
        return np.argsort(-v, kind="stable")
    if which == "sm":
        return np.argsort(np.abs(v), kind="stable")
    if which in ("lm", "sai"):
        return np.argsort(-np.abs(v), kind="stable")
    return np.arange(v.size)


def select_ritz_indices(values: np.ndarray, which: str) -> np.ndarray:
    """lanczos_select_ritz_indices (src/core/RitzExtraction.cpp:162-179), incl. BE."""
    m = values.size
    if which == "be":
        idx = []
        for i in range(m // 2):
            idx.append(m - 1 - i)
            idx.append(i)
        if m % 2 == 1:
            idx.append(m // 2)
        return np.asarray(idx, dtype=np.int64)
    return sort_indices(values, which)


@dataclass
class RitzPairs:
    values: np.ndarray
    relative_residuals: np.ndarray
    coefficients: np.ndarray
    vectors: np.ndarray
    operator_vectors: np.ndarray
    residuals: np.ndarray


def extract_projected_ritz_pairs(projected: np.ndarray, basis: np.ndarray,
                                 operator_basis: np.ndarray, active: int, requested: int,
                                 which: str, norms=None) -> RitzPairs:
    """extract_projected_ritz_pairs (src/core/RitzExtraction.cpp:65-141). ``norms``
    (optional) returns (||AXr - Xr diag(vals)||, ||Xr||) per column without forming
    the residual block, which is then not returned."""
    m = active
    P = projected[:m, :m]
    P = 0.5 * (P + P.T)
    w, Z = np.linalg.eigh(P)
    idx = select_ritz_indices(w, which)[:requested]
    vals = w[idx]
    C = Z[:, idx]
    Xr = basis[:, :m] @ C
    AXr = operator_basis[:, :m] @ C
    if norms is not None:
        Rs = None
        rn, xn = norms(AXr, Xr, vals)
    else:
        Rs = AXr - Xr * vals[None, :]
        rn = np.linalg.norm(Rs, axis=0)
        xn = np.linalg.norm(Xr, axis=0)
    den = (1.0 + np.abs(vals)) * xn
    rel = np.where(den > 0.0, rn / np.where(den > 0.0, den, 1.0), rn)
    return RitzPairs(vals, rel, C, Xr, AXr, Rs)


def evaluate_ritz_pairs(A: Csr, B: Optional[Csr], basis: np.ndarray, active: int,
                        lam: np.ndarray, Csel: np.ndarray):
    """evaluate_ritz_pairs (src/core/RitzExtraction.cpp:34-63): returns (Y, rel)."""
    Y = basis[:, :active] @ Csel
    AY = A.scipy() @ Y
    BY = (B.scipy() @ Y) if B is not None else Y.copy()
    bn = np.linalg.norm(BY, axis=0)
    R = AY - BY * lam[None, :]
    res = np.linalg.norm(R, axis=0)
    den = (1.0 + np.abs(lam)) * bn
    if np.any(~(den > 0.0)) or not np.all(np.isfinite(den)) or not np.all(np.isfinite(res)):
        raise RuntimeError("evaluate_ritz_pairs: invalid vector or non-finite residual.")
    return Y, res / den


def residual_norms(A: Csr, B: Optional[Csr], lam: np.ndarray, X: np.ndarray) -> np.ndarray:
    """fasteig_solver::compute_residual_norms (src/fasteig_solver.cpp:89-129):
    ||Ax - l Bx|| / ((1+|l|) ||Bx||) (B = I when absent)."""
    AX = A.scipy() @ X
    BX = (B.scipy() @ X) if B is not None else X
    num = np.linalg.norm(AX - BX * lam[None, :], axis=0)
    den = (1.0 + np.abs(lam)) * np.linalg.norm(BX, axis=0)
    return np.where(den > 0.0, num / np.where(den > 0.0, den, 1.0), num)


def residual_norms_baseline_def(A: Csr, B: Optional[Csr], lam: np.ndarray,
                                X: np.ndarray) -> np.ndarray:
    """The second residual definition reported beside the reference one:
    ||Kx - l Mx|| / (|l| ||Mx||)."""
    AX = A.scipy() @ X
    BX = (B.scipy() @ X) if B is not None else X
    num = np.linalg.norm(AX - BX * lam[None, :], axis=0)
    den = np.abs(lam) * np.linalg.norm(BX, axis=0)
    return np.where(den > 0.0, num / np.where(den > 0.0, den, 1.0), num)


# --------------------------------------------------------------------------
# Lanczos / Krylov subspace: src/core/KrylovSubspace.cpp:112-259,
# src/core/LanczosWorkspace.cpp:25-107
# --------------------------------------------------------------------------


class _Lanczos:
    """Scalar Lanczos with two-pass classical reorthogonalization, as built by
    KrylovSubspace::build_one (src/core/KrylovSubspace.cpp:125-131) and recorded by
    CpuLanczosWorkspace::record_step (src/core/LanczosWorkspace.cpp:25-40)."""

    def __init__(self, A_apply, residual: np.ndarray, m: int, restart_seed: int,
                 B_apply=None):
        self.A_apply = A_apply
        self.B_apply = B_apply
        self.f = residual.copy()
        self.n = residual.size
        self.V = np.zeros((self.n, m))
        self.BV = np.zeros((self.n, m)) if B_apply is not None else None
        self.Bf = None
        self.T = np.zeros((m, m))
        self.beta_next = 0.0
        self.restart_row = -1
        self.seed = restart_seed
        self.restarted = False

    def residual_norm(self) -> float:
        """KrylovSubspace::residual_norm (src/core/KrylovSubspace.cpp:162-178)."""
        if self.B_apply is not None:
            self.Bf = self.B_apply(self.f)
            sq = float(self.f @ self.Bf)
            if not math.isfinite(sq) or sq < 0.0:
                raise RuntimeError("B must be positive definite (invalid B-norm).")
            return math.sqrt(sq)
        return float(np.linalg.norm(self.f))

    def orthogonalize(self, k: int, src: np.ndarray) -> tuple[np.ndarray, float]:
        """CpuMultiVector::orthogonalize_active_columns (src/core/MultiVector.cpp:153-185)."""
        if k == 0:
            return src.copy(), 0.0
        Vk = self.V[:, :k]
        W = self.BV[:, :k] if self.BV is not None else Vk
        h = W.T @ src
        r = src - Vk @ h
        s = W.T @ r
        r = r - Vk @ s
        h = h + s
        return r, float(h[k - 1])

    def normalize_or_restart(self, it: int) -> float:
        """src/core/KrylovSubspace.cpp:232-259."""
        self.restarted = False
        beta = self.residual_norm()
        if not math.isfinite(beta):
            raise RuntimeError("non-finite residual norm encountered.")
        if beta > EPS:
            return beta
        cand = random_vector(self.n, self.seed + it + 1)
        self.f, _ = self.orthogonalize(it, cand)
        self.restarted = True
        beta = self.residual_norm()
        if beta <= EPS:
            raise RuntimeError("breakdown, unable to generate new basis vector.")
        return beta

    def step(self, it: int) -> None:
        beta = self.normalize_or_restart(it)
        self.f = self.f / beta
        self.V[:, it] = self.f
        if self.BV is not None:
            self.BV[:, it] = self.Bf / beta
        rec_beta = 0.0 if self.restarted else beta
        w = self.A_apply(self.V[:, it])
        self.f, alpha = self.orthogonalize(it + 1, w)
        beta_next = self.residual_norm()
        if not math.isfinite(beta_next):
            raise RuntimeError("non-finite next residual norm encountered.")
        self.record(it, rec_beta, alpha, beta_next)

    def record(self, it, beta, alpha, beta_next):
        if it != 0 and it != self.restart_row:
            self.T[it, it - 1] = beta
            self.T[it - 1, it] = beta
        self.T[it, it] = alpha
        self.beta_next = beta_next
        if it == self.restart_row:
            self.restart_row = -1

    def snapshot(self, m: int, nev: int, which: str):
        """lanczos_compute_cpu_snapshot + lanczos_make_snapshot_from_eigendecomp
        (src/core/RitzExtraction.cpp:181-217,252-266)."""
        w, Z = np.linalg.eigh(self.T[:m, :m])
        idx = select_ritz_indices(w, which)[:min(nev, m)]
        lam = w[idx]
        rel = np.abs(self.beta_next * Z[m - 1, idx]) / (1.0 + np.abs(lam))
        return lam, rel, Z[:, idx]


def estimate_bounds(A_apply, n: int, seed: int) -> tuple[float, float]:
    """estimate_bounds_with_executor (src/ChebyshevSolver.cpp:26-49) with
    lanczos_absolute_residuals (src/core/RitzExtraction.cpp:435-441)."""
    steps = min(20, n)
    lz = _Lanczos(A_apply, random_vector(n, seed), steps, seed)
    for it in range(steps):
        lz.step(it)
    lam, rel, _ = lz.snapshot(steps, steps, "sr")
    r = rel * (1.0 + np.abs(lam))
    lower = float((lam - r).min())
    upper = float((lam + r).max())
    if not (math.isfinite(lower) and math.isfinite(upper)) or lower > upper:
        raise RuntimeError("ChebyshevSolver: invalid spectral bound estimates.")
    return lower, upper


# --------------------------------------------------------------------------
# Solvers
# --------------------------------------------------------------------------


@dataclass
class SolveResult:
    eigenvalues: np.ndarray
    eigenvectors: np.ndarray
    residual_norms: np.ndarray
    iterations: int
    status: int = 0
    history: list = field(default_factory=list)


def chebyshev_filter_coefficients(lower: float, upper: float, degree: int):
    """Filter scaling of ChebyshevSolver::chebyshev_filter (src/ChebyshevSolver.cpp:231-239).
    Returns (c, d) of the mapped operator c*H + d*I, or None for a collapsed spectrum."""
    if upper == lower:
        return None
    amplification = 1.0e3
    xlb = math.cosh(math.acosh(amplification) / degree)
    cutoff = (2.0 * lower + upper * (xlb - 1.0)) / (1.0 + xlb)
    c = 2.0 / (upper - cutoff)
    d = -(upper + cutoff) / (upper - cutoff)
    if not (math.isfinite(c) and math.isfinite(d)):
        raise RuntimeError("ChebyshevSolver: invalid filter scaling.")
    return c, d


def chebyshev_filter(H_apply, X: np.ndarray, degree: int, lower: float, upper: float) -> np.ndarray:
    """ChebyshevSolver::chebyshev_filter (src/ChebyshevSolver.cpp:223-258):
    Y0 = X, Y1 = (cH + dI) X, Yk = 2 (cH + dI) Y_{k-1} - Y_{k-2}."""
    cd = chebyshev_filter_coefficients(lower, upper, degree)
    if cd is None:
        return X
    c, d = cd
    prev = X
    cur = c * H_apply(X) + d * X
    for _ in range(2, degree + 1):
        nxt = 2.0 * c * H_apply(cur) + 2.0 * d * cur - prev
        prev, cur = cur, nxt
    return cur


def chebyshev_filter_window(H_apply, X: np.ndarray, degree: int, cutoff: float,
                            upper: float) -> np.ndarray:
    """Three-term filter damping [cutoff, upper] into [-1, 1] (adaptive-interval
    extension; same recurrence as src/ChebyshevSolver.cpp:243-256)."""
    if upper <= cutoff:
        return X
    c = 2.0 / (upper - cutoff)
    d = -(upper + cutoff) / (upper - cutoff)
    prev = X
    cur = c * H_apply(X) + d * X
    for _ in range(2, degree + 1):
        nxt = 2.0 * c * H_apply(cur) + 2.0 * d * cur - prev
        prev, cur = cur, nxt
    return cur


def grouped_chebyshev_member(A: Csr, nev: int, degree: int = 10, tol: float = 1e-8,
                             maxiter: int = 1000, which: str = "sr", seed: int = 1,
                             block: Optional[int] = None, bounds: str = "reference",
                             amplification: float = 1e3) -> SolveResult:
    """One member of the grouped Chebyshev engine (an extension; each member runs the
    cycle of ChebyshevSolver::solve, src/ChebyshevSolver.cpp:145-205): a subspace of the
    solve's capacity (nev + min(nev, n - nev), or block) rounded up to a multiple of 32
    columns, started from the reference's seeded random block and filtered whole every
    cycle (no initial QR, no locking); the reference's filter on its Lanczos bounds
    (bounds=reference) or damped to the largest Ritz value of the subspace, capped at the
    requested amplification (bounds=ritz); Cholesky QR twice; Rayleigh-Ritz with
    W = A Y; the reference's relative residuals; done when the first nev are <= tol or at
    maxiter. FP64 (the engine's FP64 groups)."""
    n = A.rows
    which = which.lower()
    if which not in ("sr", "lr"):
        raise ValueError("grouped Chebyshev: only SR and LR are supported.")
    sign = -1.0 if which == "lr" else 1.0
    cap = nev + min(nev, n - nev) if not block else max(nev, min(block, n))
    width = (cap + 31) // 32 * 32
    if width > n:
        raise ValueError("grouped Chebyshev: width exceeds n")
    ops = NumpyChebyshevOps(A, sign)
    lower, upper = estimate_bounds(ops.apply, n, seed)

    def ref_cutoff(amp):
        xlb = math.cosh(math.acosh(amp) / degree)
        return (2.0 * lower + upper * (xlb - 1.0)) / (1.0 + xlb)

    cutoff = ref_cutoff(1e3)
    cap_cut = ref_cutoff(amplification) if bounds == "ritz" else None
    X = random_block(n, width, seed)
    for it in range(1, maxiter + 1):
        Y = X if upper == cutoff else chebyshev_filter_window(ops.apply, X, degree, cutoff, upper)
        for _ in range(2):
            info, Y, _ = cholesky_qr(Y)
            if info != 0:
                raise RuntimeError("ChebyshevSolver: Cholesky QR failed during filtering.")
        W = ops.apply(Y)
        H = Y.T @ W
        theta, Q = np.linalg.eigh(0.5 * (H + H.T))
        X = Y @ Q
        AX = W @ Q
        rel = np.linalg.norm(AX - X * theta, axis=0) / ((1.0 + np.abs(theta)) *
                                                         np.linalg.norm(X, axis=0))
        if rel[:nev].max() <= tol or it == maxiter:
            return SolveResult(sign * theta[:nev], X[:, :nev], rel[:nev], it,
                               0 if rel[:nev].max() <= tol else 1)
        if cap_cut is not None:
            cutoff = min(theta[-1], cap_cut)
    raise RuntimeError("grouped Chebyshev: unreachable")


class NumpyChebyshevOps:
    """Operator applications of the Chebyshev loop with SciPy/NumPy (the parity path)."""

    def __init__(self, A: Csr, sign: float):
        self.Hs = A.scipy()
        self.sign = sign

    def apply(self, X: np.ndarray) -> np.ndarray:
        return self.sign * (self.Hs @ X)

    def filter(self, X: np.ndarray, degree: int, lower: float, upper: float) -> np.ndarray:
        return chebyshev_filter(self.apply, X, degree, lower, upper)

    def filter_window(self, X: np.ndarray, degree: int, cutoff: float, upper: float) -> np.ndarray:
        return chebyshev_filter_window(self.apply, X, degree, cutoff, upper)


@dataclass
class ChebyshevProgress:
    """State after one cycle of chebyshev_cycles."""
    iteration: int = 0
    locked: int = 0
    filtered_cols: int = 0
    worst: float = math.inf
    converged: bool = False
    result: Optional[SolveResult] = None


def chebyshev_solve(A: Csr, nev: int, degree: int = 10, tol: float = 1e-8,
                    maxiter: int = 1000, which: str = "sr", seed: int = 1,
                    block: Optional[int] = None, record_history: bool = False,
                    bounds: str = "reference", amplification: float = math.inf,
                    locking: str = "soft", ops=None,
                    v0: Optional[np.ndarray] = None) -> SolveResult:
    """ChebyshevSolver::solve (src/ChebyshevSolver.cpp:67-221); runs
    chebyshev_cycles to the end and returns its result."""
    prog = None
    for prog in chebyshev_cycles(A, nev, degree, tol, maxiter, which, seed, block,
                                 record_history, bounds, amplification, locking, ops, v0):
        pass
    return prog.result


def chebyshev_cycles(A: Csr, nev: int, degree: int = 10, tol: float = 1e-8,
                     maxiter: int = 1000, which: str = "sr", seed: int = 1,
                     block: Optional[int] = None, record_history: bool = False,
                     bounds: str = "reference", amplification: float = math.inf,
                     locking: str = "soft", ops=None, v0: Optional[np.ndarray] = None):
    """ChebyshevSolver::solve (src/ChebyshevSolver.cpp:67-221), one filter cycle per
    ``next()``: the first call also runs the set-up (random block, Cholesky QR,
    Lanczos bounds). Yields a ChebyshevProgress after every cycle; the last one
    carries the SolveResult.

    ``block`` overrides the subspace capacity ``nev + min(nev, n - nev)``
    (src/ChebyshevSolver.cpp:94); None keeps the reference behaviour.
    ``bounds="ritz"`` is the adaptive-interval extension (not in the reference):
    after each Rayleigh-Ritz the damped interval is [theta_max, upper], where
    theta_max is the largest Ritz value of the subspace (Zhou & Saad, 2007), and
    the cutoff is lowered where needed so that the filter's amplification at
    the Lanczos lower bound stays within ``amplification``.
    ``locking="hard"`` is the hard-locking extension (not in the reference, which
    rechecks the whole prefix after a Rayleigh-Ritz over the whole subspace,
    src/ChebyshevSolver.cpp:160-192): locked pairs are final, and the QR and the
    Rayleigh-Ritz act on the deflated active block only; pairs are returned in
    ascending order.
    ``ops`` applies the operator (NumpyChebyshevOps by default; oracle/cpu.py has a
    threaded host version with the same arithmetic for timing at full size)."""
    n = A.rows
    which = which.lower()
    if n <= 0 or nev <= 0 or nev > n:
        raise ValueError("ChebyshevSolver: nev must be in [1,n].")
    if which not in ("sr", "lr"):
        raise ValueError("ChebyshevSolver: only SR and LR are supported.")
    sign = -1.0 if which == "lr" else 1.0
    if ops is None:
        ops = NumpyChebyshevOps(A, sign)
    H_apply = ops.apply
    norms = getattr(ops, "residual_norms", None)
    capacity = nev + min(nev, n - nev) if block is None else max(nev, min(block, n))
    vectors = warm_start(random_block(n, capacity, seed), v0, nev, "ChebyshevSolver")
    info, vectors, _ = cholesky_qr(vectors)
    if info != 0:
        raise RuntimeError("ChebyshevSolver: initial Cholesky QR failed.")
    lower, upper = estimate_bounds(lambda v: H_apply(v), n, seed)

    locked = 0
    subspace_cols = nev
    ritz = None
    it_done = 0
    history = []
    prog = ChebyshevProgress()
    for it in range(maxiter):
        active = subspace_cols - locked
        if bounds == "ritz" and ritz is not None:
            cutoff = float(ritz.values[-1] if locking == "hard"
                           else ritz.values[subspace_cols_prev - 1])
            if math.isfinite(amplification):
                xl = math.cosh(math.acosh(amplification) / degree)
                cutoff = min(cutoff, (2.0 * lower + upper * (xl - 1.0)) / (1.0 + xl))
            filtered = ops.filter_window(vectors[:, locked:locked + active].copy(), degree,
                                         cutoff, upper)
        else:
            filtered = ops.filter(vectors[:, locked:locked + active].copy(), degree, lower, upper)
        if locked > 0:
            _, filtered, _ = block_gram_schmidt(vectors, locked, filtered)
        vectors[:, locked:locked + active] = filtered
        prog.filtered_cols = active
        if locking == "hard":
            info, basis, _ = cholesky_qr(filtered)
            if info != 0:
                raise RuntimeError("ChebyshevSolver: Cholesky QR failed during filtering.")
            op_basis = H_apply(basis)
            ritz_a = extract_projected_ritz_pairs(basis.T @ op_basis, basis, op_basis, active,
                                                  active, "sr", norms)
            del basis, op_basis
            if ritz is None:
                vals, rels = np.zeros(capacity), np.zeros(capacity)
            vals[locked:subspace_cols] = ritz_a.values
            rels[locked:subspace_cols] = ritz_a.relative_residuals
            if not (np.all(np.isfinite(ritz_a.values)) and
                    np.all(np.isfinite(ritz_a.relative_residuals))):
                raise RuntimeError("ChebyshevSolver: non-finite Ritz values or residuals.")
            vectors[:, locked:subspace_cols] = ritz_a.vectors
            ritz = RitzPairs(ritz_a.values, ritz_a.relative_residuals, ritz_a.coefficients,
                             None, None, None)
            del ritz_a
            subspace_cols_prev = subspace_cols
            while locked < nev and rels[locked] <= tol:
                locked += 1
            subspace_cols = max(subspace_cols, nev + min(locked, capacity - nev))
            it_done = it + 1
            if record_history:
                history.append((sign * vals[:nev].copy(), rels[:nev].copy()))
            prog.iteration, prog.locked, prog.worst = it_done, locked, float(rels[:nev].max())
            if rels[:nev].max() <= tol:
                prog.converged = True
                break
            yield prog
            continue
        basis = vectors[:, :subspace_cols].copy()
        info, basis, _ = cholesky_qr(basis)
        if info != 0:
            raise RuntimeError("ChebyshevSolver: Cholesky QR failed during filtering.")
        op_basis = H_apply(basis)
        projected = basis.T @ op_basis
        ritz = extract_projected_ritz_pairs(projected, basis, op_basis, subspace_cols,
                                            subspace_cols, "sr", norms)
        if not (np.all(np.isfinite(ritz.values)) and np.all(np.isfinite(ritz.relative_residuals))):
            raise RuntimeError("ChebyshevSolver: non-finite Ritz values or residuals.")
        vectors[:, :subspace_cols] = ritz.vectors
        subspace_cols_prev = subspace_cols
        locked = 0
        while locked < nev and ritz.relative_residuals[locked] <= tol:
            locked += 1
        subspace_cols = max(subspace_cols, nev + min(locked, capacity - nev))
        it_done = it + 1
        if record_history:
            history.append((sign * ritz.values[:nev].copy(), ritz.relative_residuals[:nev].copy()))
        prog.iteration, prog.locked = it_done, locked
        prog.worst = float(ritz.relative_residuals[:nev].max())
        if ritz.relative_residuals[:nev].max() <= tol:
            prog.converged = True
            break
        yield prog
    if locking == "hard":
        order = np.argsort(vals[:nev], kind="stable")
        prog.result = SolveResult(sign * vals[:nev][order], vectors[:, :nev][:, order].copy(),
                                  rels[:nev][order].copy(), it_done, 0, history)
    else:
        prog.result = SolveResult(sign * ritz.values[:nev], ritz.vectors[:, :nev].copy(),
                                  ritz.relative_residuals[:nev].copy(), it_done, 0, history)
    yield prog


def lobpcg_solve(A: Csr, nev: int, tol: float = 1e-8, maxiter: int = 1000,
                 which: str = "sr", seed: int = 1,
                 v0: Optional[np.ndarray] = None) -> SolveResult:
    """LOBPCGSolver::solve (src/LOBPCGSolver.cpp:25-174): unpreconditioned LOBPCG,
    block width nev, soft locking."""
    n = A.rows
    which = which.lower()
    if n <= 0 or nev <= 0 or nev > n or maxiter <= 0:
        raise ValueError("LOBPCGSolver: require 0 < nev <= n and maxiter > 0.")
    if which not in ("sr", "lr"):
        raise ValueError("LOBPCGSolver: only SR and LR are supported.")
    sign = -1.0 if which == "lr" else 1.0
    Hs = A.scipy()
    H_apply = (lambda X: sign * (Hs @ X))
    X = warm_start(random_block(n, nev, seed), v0, nev, "LOBPCGSolver")
    _, X, _ = householder_qr(X)
    capacity = min(n, 3 * nev)
    AX = H_apply(X)
    ritz = extract_projected_ritz_pairs(X.T @ AX, X, AX, nev, nev, "sr")
    X = ritz.vectors
    P = None
    it_done = 0
    for it in range(maxiter):
        if not (np.all(np.isfinite(ritz.values)) and np.all(np.isfinite(ritz.relative_residuals))):
            raise RuntimeError("LOBPCGSolver: non-finite Ritz values or residuals.")
        if ritz.relative_residuals.max() <= tol:
            break
        active = [j for j in range(nev) if ritz.relative_residuals[j] > tol]
        W_source = ritz.residuals[:, active]
        _, X, _ = householder_qr(X)
        basis = np.zeros((n, capacity))
        basis[:, :nev] = X
        cols = nev
        W = orthonormalize_block(basis, cols, W_source)
        if W is not None:
            basis[:, cols:cols + W.shape[1]] = W
            cols += W.shape[1]
        if P is not None and cols < capacity:
            Po = orthonormalize_block(basis, cols, P[:, active])
            if Po is not None:
                take = Po.shape[1]
                basis[:, cols:cols + take] = Po
                cols += take
        op_basis = H_apply(basis[:, :cols])
        projected = basis[:, :cols].T @ op_basis
        ritz = extract_projected_ritz_pairs(projected, basis, op_basis, cols, nev, "sr")
        if not (np.all(np.isfinite(ritz.values)) and np.all(np.isfinite(ritz.relative_residuals))):
            raise RuntimeError("LOBPCGSolver: non-finite Ritz values or residuals.")
        dc = ritz.coefficients.copy()
        dc[:nev, :] = 0.0
        P = basis[:, :cols] @ dc
        X = ritz.vectors
        it_done = it + 1
        if ritz.relative_residuals.max() <= tol or cols == nev:
            break
    return SolveResult(sign * ritz.values, X.copy(), ritz.relative_residuals.copy(), it_done)


def davidson_solve(A: Csr, nev: int, tol: float = 1e-8, maxiter: int = 1000,
                   which: str = "sr", seed: int = 1, maxblks: int = 10,
                   v0: Optional[np.ndarray] = None) -> SolveResult:
    """DavidsonSolver::solve (src/DavidsonSolver.cpp:27-264): block Davidson with thick
    restart and unpreconditioned corrections; locktol = min(1e-5, tol) (:126)."""
    n = A.rows
    which = which.lower()
    if nev <= 0 or nev > n:
        raise ValueError("DavidsonSolver: nev must be in [1,n].")
    Hs = A.scipy()
    H_apply = (lambda X: Hs @ X)
    V0 = warm_start(random_block(n, nev, seed), v0, nev, "DavidsonSolver")
    info, V0, _ = cholesky_qr(V0)
    if info != 0:
        raise RuntimeError("DavidsonSolver: initial Cholesky QR failed.")
    max_cols = min(n, maxblks * nev)
    AV0 = H_apply(V0)
    ritz = extract_projected_ritz_pairs(V0.T @ AV0, V0, AV0, nev, nev, which)
    locktol = min(1.0e-5, tol)
    it_done = 0
    for it in range(maxiter):
        _, Xr, _ = householder_qr(ritz.vectors)
        AXr = H_apply(Xr)
        basis = np.zeros((n, max_cols))
        op_basis = np.zeros((n, max_cols))
        basis[:, :nev] = Xr
        op_basis[:, :nev] = AXr
        projected = np.zeros((max_cols, max_cols))
        projected[:nev, :nev] = Xr.T @ AXr
        cols = nev
        ritz = extract_projected_ritz_pairs(projected, basis, op_basis, nev, nev, which)
        for _blk in range(1, maxblks):
            active = [j for j in range(nev) if ritz.relative_residuals[j] > locktol]
            cc = len(active)
            if cc == 0 or cols + cc > max_cols:
                break
            src = ritz.residuals[:, active]
            _, corr, _ = block_gram_schmidt(basis, cols, src)
            _, corr, _ = householder_qr(corr)
            Acorr = H_apply(corr)
            cross = basis[:, :cols].T @ Acorr
            diag = corr.T @ Acorr
            diag = 0.5 * (diag + diag.T)
            projected[:cols, cols:cols + cc] = cross
            projected[cols:cols + cc, :cols] = cross.T
            projected[cols:cols + cc, cols:cols + cc] = diag
            basis[:, cols:cols + cc] = corr
            op_basis[:, cols:cols + cc] = Acorr
            cols += cc
            ritz = extract_projected_ritz_pairs(projected, basis, op_basis, cols, nev, which)
        it_done = it + 1
        if ritz.relative_residuals.size > 0 and ritz.relative_residuals.max() < tol:
            break
    return SolveResult(ritz.values.copy(), ritz.vectors.copy(),
                       ritz.relative_residuals.copy(), it_done)


def krylov_schur_solve(A: Csr, nev: int, tol: float = 1e-8, maxiter: int = 1000,
                       which: str = "sr", seed: int = 1, maxdim: int = 0,
                       B: Optional[Csr] = None, v0: Optional[np.ndarray] = None) -> SolveResult:
    """KrylovSchurSolver::solve (src/KrylovSchurSolver.cpp:28-160), standard problems
    (B is None) and the B-metric Lanczos of src/core/KrylovSubspace.cpp:162-178 with an
    explicit B^{-1}A operator for generalized problems (the reference's cuDSS/LU
    factorization is replaced by a sparse direct solve here)."""
    n = A.rows
    which = which.lower()
    m = min(max(2 * nev, 20, maxdim), n)
    Hs = A.scipy()
    if B is None:
        A_apply = (lambda v: Hs @ v)
        B_apply = None
    else:
        import scipy.sparse.linalg as spla
        lu = spla.splu(B.scipy().tocsc())
        Bs = B.scipy()
        A_apply = (lambda v: lu.solve(Hs @ v))
        B_apply = (lambda v: Bs @ v)
    start = random_vector(n, seed) if v0 is None else \
        warm_start(np.zeros((n, 1)), v0, 1, "KrylovSchurSolver")[:, 0]  # v0.col(0) (:68-70)
    lz = _Lanczos(A_apply, start, m, seed, B_apply)
    for col in range(m):
        lz.step(col)
    for it in range(1, maxiter + 1):
        w, Z = np.linalg.eigh(lz.T[:m, :m])
        idx = select_ritz_indices(w, which)
        lam_all = w[idx]
        C_all = Z[:, idx]
        rel_all = np.abs(lz.beta_next * Z[m - 1, idx]) / (1.0 + np.abs(lam_all))
        nconv = 0
        for j in range(nev):
            mag = abs(lam_all[j])
            ok = (rel_all[j] <= tol) if B is not None else (rel_all[j] * (1.0 + mag) < tol * mag)
            nconv += int(ok)
        at_limit = (m == n) or (it == maxiter)
        if nconv >= nev or at_limit:
            Y, res = evaluate_ritz_pairs(A, B, lz.V, m, lam_all[:nev], C_all[:, :nev])
            verified = bool(np.all(res <= tol))
            if B is None or verified or at_limit:
                status = 1 if (B is not None and not verified) else 0
                return SolveResult(lam_all[:nev].copy(), Y, res, it, status)
        spare = (m - nev) // 2
        retained = nev + min(nconv, spare)
        if retained == 1 and m > 3:
            retained = m // 2
        C = C_all[:, :retained]
        lz.V[:, :retained] = lz.V[:, :m] @ C
        if lz.BV is not None:
            lz.BV[:, :retained] = lz.BV[:, :m] @ C
        T = np.zeros_like(lz.T)
        for j in range(retained):
            T[j, j] = lam_all[j]
            cpl = lz.beta_next * C_all[m - 1, j]
            T[retained, j] = cpl
            T[j, retained] = cpl
        lz.T = T
        lz.restart_row = retained
        for col in range(retained, m):
            lz.step(col)
    raise RuntimeError("KrylovSchurSolver: unreachable solve termination.")


def lanczos_solve(A: Csr, nev: int, tol: float = 1e-8, maxiter: int = 1000,
                  which: str = "sr", seed: int = 1, print_every: int = 0,
                  B: Optional[Csr] = None, v0: Optional[np.ndarray] = None) -> SolveResult:
    """LanczosSolver::solve (src/LanczosSolver.cpp:29-163): one scalar Lanczos chain of up
    to maxiter vectors, no restart; from nev vectors on, every check_every-th step
    (print_every, else 5) and at maxiter the projected tridiagonal is diagonalized and
    the chain stops when every wanted estimate |beta_m z_{m-1,j}| / (1 + |theta_j|) is
    below tol (B metric: the formed pairs must pass their residual check too, and a
    chain that broke down keeps going to recover multiplicity). Generalized problems
    use the B^-1 A operator of krylov_schur_solve."""
    n = A.rows
    which = which.lower()
    if maxiter <= 0:
        raise ValueError("LanczosSolver: maxiter must be > 0.")
    if nev <= 0:
        raise ValueError("LanczosSolver: nev must be > 0.")
    if maxiter < nev:
        raise ValueError("LanczosSolver: maxiter must be >= nev.")
    if maxiter > n:
        raise ValueError("LanczosSolver: maxiter must be <= n.")
    Hs = A.scipy()
    if B is None:
        A_apply, B_apply = (lambda v: Hs @ v), None
    else:
        import scipy.sparse.linalg as spla
        lu = spla.splu(B.scipy().tocsc())
        Bs = B.scipy()
        A_apply = (lambda v: lu.solve(Hs @ v))
        B_apply = (lambda v: Bs @ v)
    start = random_vector(n, seed) if v0 is None else \
        warm_start(np.zeros((n, 1)), v0, 1, "LanczosSolver")[:, 0]  # v0.col(0)
    lz = _Lanczos(A_apply, start, maxiter, seed, B_apply)
    check_every = print_every if print_every > 0 else 5
    breakdown = False
    for it in range(maxiter):
        beta_prev = lz.T[it, it - 1] if it > 0 else 0.0
        lz.step(it)
        alpha = lz.T[it, it]
        breakdown = breakdown or lz.beta_next <= 64.0 * EPS * max(1.0, abs(alpha), abs(beta_prev))
        m = it + 1
        if not (m >= nev and (m % check_every == 0 or m == maxiter)):
            continue
        resolve_multiplicity = B is not None and breakdown and m < maxiter
        lam, rel, C = lz.snapshot(m, nev, which)
        if not resolve_multiplicity and rel.max() < tol:
            Y, res = evaluate_ritz_pairs(A, B, lz.V, m, lam, C)
            if B is not None and not np.all(res <= tol):
                continue
            return SolveResult(lam.copy(), Y, res, m, 0)
    lam, rel, C = lz.snapshot(maxiter, nev, which)
    Y, res = evaluate_ritz_pairs(A, B, lz.V, maxiter, lam, C)
    status = 1 if (B is not None and not np.all(res <= tol)) else 0
    return SolveResult(lam.copy(), Y, res, maxiter, status)


def _cgs2(V: np.ndarray, k: int, src: np.ndarray) -> np.ndarray:
    """Two-pass classical Gram-Schmidt of one vector against V[:, :k]
    (CpuMultiVector::orthogonalize_active_columns, src/core/MultiVector.cpp:153-185)."""
    if k == 0:
        return src.copy()
    Vk = V[:, :k]
    r = src - Vk @ (Vk.T @ src)
    return r - Vk @ (Vk.T @ r)


def complete_block_qr(basis: np.ndarray, active_cols: int, source: np.ndarray, seed: int,
                      reference_norm: float):
    """complete_block_qr (src/core/Orthogonalization.cpp:609-715), standard inner product.
    Returns (replenished, Q, R)."""
    n, b = source.shape
    capacity = min(b, n - active_cols)
    threshold = 64.0 * EPS * reference_norm
    if capacity == b:
        info, Q, R = cholesky_qr(source.copy())
        if info == 0:
            gram = Q.T @ Q
            cross = basis[:, :active_cols].T @ Q
            if (np.all(np.isfinite(R)) and np.abs(np.diag(R)).min() > threshold and
                    np.all(np.isfinite(gram)) and np.all(np.isfinite(cross)) and
                    np.linalg.norm(gram - np.eye(b)) < 1e-10 and np.linalg.norm(cross) < 1e-10):
                return False, Q, R
    replenished = False
    Q = np.zeros((n, b))

    def project(v, j):
        return _cgs2(Q, j, _cgs2(basis, active_cols, v))

    for j in range(capacity):
        length, original_scale, best = 0.0, 0.0, None
        for col in range(b):
            v = source[:, col].copy()
            original_scale = max(original_scale, float(np.linalg.norm(v)))
            v = project(v, j)
            cn = float(np.linalg.norm(v))
            if cn > length:
                length, best = cn, v.copy()
        cutoff = max(threshold, 1e-12 * original_scale)
        if length > cutoff:
            v = best
            length = float(np.linalg.norm(v))
        if not (length > cutoff):
            replenished = True
            length = 0.0
            for attempt in range(4):
                v = random_vector(n, seed + 17 * (j + 1) + attempt)
                rn = float(np.linalg.norm(v))
                v = project(v, j)
                length = float(np.linalg.norm(v))
                if length > 1e-12 * rn:
                    break
                length = 0.0
            if length == 0.0:
                raise RuntimeError("complete_block_qr: unable to complete the basis.")
        Q[:, j] = v / length
    R = Q.T @ source
    R[:, np.linalg.norm(R, axis=0) <= threshold] = 0.0
    return replenished, Q, R


def block_krylov_schur_solve(A: Csr, nev: int, blksize: int, tol: float = 1e-8,
                             maxiter: int = 1000, which: str = "sr", seed: int = 1,
                             maxdim: int = 0, v0: Optional[np.ndarray] = None) -> SolveResult:
    """BlockKrylovSchurSolver::solve (src/BlockKrylovSchurSolver.cpp:26-215) for standard
    problems: BlockKrylovSubspace expansion (src/core/KrylovSubspace.cpp:261-437: block
    apply, two-pass block Gram-Schmidt, complete_block_qr of the residual block),
    block-tridiagonal projection (src/core/LanczosWorkspace.cpp:42-73), Ritz residual
    estimates from the coupling block (src/core/RitzExtraction.cpp:272-380) and the thick
    block restart (src/core/LanczosWorkspace.cpp:109-135)."""
    n = A.rows
    which = which.lower()
    if n <= 0:
        raise ValueError("BlockKrylovSchurSolver: n must be > 0.")
    if nev <= 0 or nev > n:
        raise ValueError("BlockKrylovSchurSolver: nev must be in [1,n].")
    if maxiter <= 0:
        raise ValueError("BlockKrylovSchurSolver: maxiter must be > 0.")
    if which not in ("sr", "lr", "sm", "lm", "be"):
        raise ValueError("BlockKrylovSchurSolver: invalid which option.")
    b = int(blksize)
    if b <= 0 or b > n:
        raise ValueError("BlockKrylovSchurSolver: blksize must be in [1,n].")
    requested_dim = maxdim if maxdim > 0 else max(2 * nev, 20)
    block_count = (1 + (n - 1) // b) if requested_dim >= n else requested_dim // b
    cycle_dim = min(n, block_count * b)
    wanted_blocks = 1 + (nev - 1) // b
    if cycle_dim < n and block_count <= wanted_blocks:
        raise ValueError("BlockKrylovSchurSolver: maxdim must accommodate ceil(nev/blksize) "
                         "retained blocks plus at least one expansion block (or the full "
                         "matrix dimension).")
    projection_dim = (block_count + 1) * b
    retained_blocks = 0 if cycle_dim == n else max(wanted_blocks, block_count // 2)
    retained_dim = retained_blocks * b
    snapshot_count = max(nev, retained_dim)
    Hs = A.scipy()
    basis = np.zeros((n, projection_dim))
    first = random_block(n, b, seed) if v0 is None else leading_block(v0, n, b, "BlockKrylovSchurSolver")
    _, Q0, _ = complete_block_qr(basis, 0, first, seed, 0.0)
    basis[:, :b] = Q0
    T = np.zeros((projection_dim, projection_dim))
    beta = np.zeros((b, b))

    def expand(first_block):
        nonlocal beta
        for block in range(first_block, block_count):
            Z = Hs @ basis[:, block * b:(block + 1) * b]
            active = min(n, (block + 1) * b)
            _, Rres, H = block_gram_schmidt(basis, active, Z)
            width = 1 + (active - 1) % b
            diag = np.zeros((b, b))
            diag[:width, :width] = H[H.shape[0] - width:, :width]
            scale = float(np.linalg.norm(np.linalg.norm(Z, axis=0)))
            _, Qn, coupling = complete_block_qr(basis, min((block + 1) * b, n), Rres,
                                                seed + (block + 1) * b, scale)
            basis[:, (block + 1) * b:(block + 2) * b] = Qn
            row, nrow = block * b, (block + 1) * b
            T[row:row + b, row:row + b] = diag
            T[nrow:nrow + b, row:row + b] = coupling
            T[row:row + b, nrow:nrow + b] = coupling.T
            beta = coupling

    expand(0)
    for iteration in range(1, maxiter + 1):
        m = cycle_dim
        w, Z = np.linalg.eigh(T[:m, :m])
        tail = 1 + (m - 1) % b
        last = np.zeros((b, m))
        last[:tail] = Z[m - tail:, :]
        idx = select_ritz_indices(w, which)
        cnt = min(snapshot_count, m)
        lam_all = w[idx[:cnt]]
        rel_all = np.linalg.norm(beta @ last[:, idx[:cnt]], axis=0) / (1.0 + np.abs(lam_all))
        C_all = Z[:, idx[:cnt]]
        k = min(nev, cnt)
        converged = k > 0 and rel_all[:k].max() < tol
        at_limit = iteration == maxiter or cycle_dim == n
        if converged or at_limit:
            Y, res = evaluate_ritz_pairs(A, None, basis, cycle_dim, lam_all[:k], C_all[:, :k])
            converged = bool(np.all(res <= tol))
            if converged or at_limit:
                return SolveResult(lam_all[:k].copy(), Y, res, iteration, 0 if converged else 1)
        Cr = C_all[:, :retained_dim]
        restart_coupling = beta @ Cr[m - b:, :]
        ritz_block = basis[:, :cycle_dim] @ Cr
        resid_block = basis[:, block_count * b:block_count * b + b].copy()
        basis[:] = 0.0
        basis[:, :retained_dim] = ritz_block
        basis[:, retained_dim:retained_dim + b] = resid_block
        T[:] = 0.0
        T[:retained_dim, :retained_dim] = np.diag(lam_all[:retained_dim])
        T[retained_dim:retained_dim + b, :retained_dim] = restart_coupling
        T[:retained_dim, retained_dim:retained_dim + b] = restart_coupling.T
        expand(retained_blocks)
    raise RuntimeError("BlockKrylovSchurSolver: unreachable solve termination.")


def block_lanczos_solve(A: Csr, nev: int, blksize: int, tol: float = 1e-8,
                        maxiter: int = 1000, which: str = "sr", seed: int = 1,
                        v0: Optional[np.ndarray] = None) -> SolveResult:
    """BlockLanczosSolver::solve (src/BlockLanczosSolver.cpp:24-176) for standard problems:
    one block Krylov chain (BlockKrylovSubspace, src/core/KrylovSubspace.cpp:261-437: the
    seeded random block, block apply, two-pass block Gram-Schmidt against the active
    basis, complete_block_qr of the residual block) of up to maxiter blocks with no
    restart; after every block from iter * blksize >= nev on, the block-tridiagonal
    projection is diagonalized and the chain stops when every wanted estimate
    ||beta y_last|| / (1 + |theta|) is below tol; the pairs are then formed from the
    basis and their residuals evaluated (evaluate_ritz_pairs)."""
    n = A.rows
    which = which.lower()
    b = int(blksize)
    if n <= 0:
        raise ValueError("BlockLanczosSolver: n must be > 0.")
    if nev <= 0:
        raise ValueError("BlockLanczosSolver: nev must be > 0.")
    if maxiter <= 0:
        raise ValueError("BlockLanczosSolver: maxiter must be > 0.")
    if b <= 0:
        raise ValueError("BlockLanczosSolver: blksize must be > 0.")
    if b > n or nev > n:
        raise ValueError("BlockLanczosSolver: blksize and nev must be <= n.")
    max_blocks = int(maxiter)
    if max_blocks * b < nev:
        raise ValueError("BlockLanczosSolver: need maxiter*blksize >= nev.")
    if which not in ("sr", "lr", "sm", "lm", "be"):
        raise ValueError("BlockLanczosSolver: invalid which option.")
    Hs = A.scipy()
    cap_blocks = min(max_blocks, 1 + (n - 1) // b, 32) + 1  # grown on demand

    basis = np.zeros((n, cap_blocks * b))
    first = random_block(n, b, seed) if v0 is None else leading_block(v0, n, b, "BlockLanczosSolver")
    _, Q0, _ = complete_block_qr(basis, 0, first, seed, 0.0)
    basis[:, :b] = Q0
    T = np.zeros((cap_blocks * b, cap_blocks * b))
    beta = np.zeros((b, b))

    def snapshot(m):
        w, Z = np.linalg.eigh(T[:m, :m])
        tail = 1 + (m - 1) % b
        last = np.zeros((b, m))
        last[:tail] = Z[m - tail:, :]
        idx = select_ritz_indices(w, which)[:min(nev, m)]
        rel = np.linalg.norm(beta @ last[:, idx], axis=0) / (1.0 + np.abs(w[idx]))
        return w[idx], rel, Z[:, idx]

    for it in range(1, max_blocks + 1):
        if (it + 1) * b > basis.shape[1]:
            grow = basis.shape[1]
            basis = np.concatenate([basis, np.zeros((n, grow))], axis=1)
            T2 = np.zeros((T.shape[0] + grow, T.shape[1] + grow))
            T2[:T.shape[0], :T.shape[1]] = T
            T = T2
        Z = Hs @ basis[:, (it - 1) * b:it * b]
        active = min(n, it * b)
        _, Rres, H = block_gram_schmidt(basis, active, Z)
        width = 1 + (active - 1) % b
        diag = np.zeros((b, b))
        diag[:width, :width] = H[H.shape[0] - width:, :width]
        scale = float(np.linalg.norm(np.linalg.norm(Z, axis=0)))
        _, Qn, coupling = complete_block_qr(basis, active, Rres, seed + it * b, scale)
        basis[:, it * b:(it + 1) * b] = Qn
        row, nrow = (it - 1) * b, it * b
        T[row:row + b, row:row + b] = diag
        T[nrow:nrow + b, row:row + b] = coupling
        T[row:row + b, nrow:nrow + b] = coupling.T
        beta = coupling
        if it * b < nev and it < max_blocks:
            continue
        lam, rel, C = snapshot(active)
        if rel.size and rel.max() < tol or it == max_blocks or active == n:
            Y, res = evaluate_ritz_pairs(A, None, basis, active, lam, C)
            return SolveResult(lam.copy(), Y, res, it, 0)
    raise RuntimeError("BlockLanczosSolver: unreachable solve termination.")


# --------------------------------------------------------------------------
# Reference spectra: tests/scripts/ref_eigs.py (parse) and run_case.py (select)
# --------------------------------------------------------------------------


def select_reference(values, which: str, count: int, shift: float = 0.0):
    """select_reference (tests/scripts/run_case.py:207-221)."""
    ordered = sorted(values)
    which = which.upper()
    if which == "SR":
        return ordered[:count]
    if which == "LR":
        return ordered[::-1][:count]
    if which == "SM":
        return sorted(ordered, key=abs)[:count]
    if which == "LM":
        return sorted(ordered, key=abs, reverse=True)[:count]
    if which == "BE":
        return [ordered[-1 - i // 2] if i % 2 == 0 else ordered[i // 2] for i in range(count)]
    if which == "SAI":
        return sorted(sorted(ordered, key=lambda v: abs(v - shift))[:count])
    raise ValueError(which)


def eigenvalue_check(got, expected, atol: float = 1e-10, rtol: float = 1e-10):
    """compare() of tests/scripts/run_case.py:246-260: |got-exp| <= atol + rtol*|exp|."""
    return [abs(g - e) <= atol + rtol * abs(e) for g, e in zip(got, expected)]


# --------------------------------------------------------------------------
# Extension (not in the reference): generalized K u = l M u and Jacobi-
# preconditioned LOBPCG / block Davidson. The reference's LOBPCGSolver and
# DavidsonSolver are standard-only and unpreconditioned (src/LOBPCGSolver.cpp:25-174,
# src/DavidsonSolver.cpp:27-264); these follow the same loop structure with every
# inner product taken in the B metric (B-weighted Gram as in the reference's
# weighted Cholesky QR, src/core/Orthogonalization.cpp:407-440), corrections
# W = T R with T = diag(|K_ii|)^-1, and the relative residual of
# evaluate_ritz_pairs with B (src/core/RitzExtraction.cpp:50-56):
# ||K x - l M x|| / ((1 + |l|) ||M x||). The CUDA drivers execute the same steps.
# --------------------------------------------------------------------------


def jacobi_inverse_diagonal(A: Csr) -> np.ndarray:
    """t_i = 1 / |A_ii| (1 where the diagonal entry is zero or absent)."""
    d = np.abs(A.scipy().diagonal())
    return np.where(d > 0.0, 1.0 / np.where(d > 0.0, d, 1.0), 1.0)


def _b_apply(B: Optional[Csr], X: np.ndarray) -> np.ndarray:
    return X.copy() if B is None else B.scipy() @ X


def ortho_block_b(B: Optional[Csr], V: Optional[np.ndarray], BV: Optional[np.ndarray], k: int,
                  source: np.ndarray, rank_tolerance: float = 1e-12):
    """B-orthonormal basis of the part of `source` outside span(V[:, :k]) (V B-orthonormal,
    BV = B V): two passes of B-norms -> two-pass block Gram-Schmidt in the B metric ->
    B-Gram eigen-decomposition -> keep singular values above
    max(rank_tolerance * largest B-norm, 1e-7 * largest singular value) -> rotate by
    U S^-1 (orthonormalize_block, src/core/Orthogonalization.cpp:717-775, with the SVD of
    the QR factor replaced by the B-Gram). Returns (Q, BQ) or (None, None)."""
    n = source.shape[0]
    if k >= n:
        return None, None
    cur = source
    BQ = None
    for _ in range(2):
        Bc = _b_apply(B, cur)
        bn = np.sqrt(np.maximum(np.sum(cur * Bc, axis=0), 0.0))
        if not np.all(np.isfinite(bn)):
            raise RuntimeError("orthonormalize_block: non-finite column norms.")
        scale = bn.max()
        if scale == 0.0:
            return None, None
        if k > 0:
            for _g in range(2):
                H = V[:, :k].T @ Bc
                cur = cur - V[:, :k] @ H
                Bc = Bc - BV[:, :k] @ H
        G = cur.T @ Bc
        G = 0.5 * (G + G.T)
        w, U = np.linalg.eigh(G)
        cols = cur.shape[1]
        smax = math.sqrt(max(w[-1], 0.0))
        cut = max(rank_tolerance * scale, 1e-7 * smax)
        capacity = min(cols, n - k)
        sel, inv = [], []
        for i in range(cols - 1, -1, -1):
            if len(sel) >= capacity:
                break
            sv = math.sqrt(max(w[i], 0.0))
            if not sv > cut:
                break
            sel.append(i)
            inv.append(1.0 / sv)
        if not sel:
            return None, None
        C = U[:, sel] * np.asarray(inv)[None, :]
        cur = cur @ C
        BQ = Bc @ C
    return cur, BQ


def b_cholesky_qr(B: Optional[Csr], X: np.ndarray):
    """Weighted Cholesky QR with a fresh BX (src/core/Orthogonalization.cpp:407-440):
    returns (X R^-1, BX R^-1)."""
    BX = _b_apply(B, X)
    G = X.T @ BX
    G = 0.5 * (G + G.T)
    try:
        L = np.linalg.cholesky(G)
    except np.linalg.LinAlgError:
        raise RuntimeError("weighted Cholesky QR failed.")
    Rinv = np.linalg.inv(L.T)
    return X @ Rinv, BX @ Rinv


def _gen_ritz(S, AS, BS, cols, req, which):
    P = S[:, :cols].T @ AS[:, :cols]
    P = 0.5 * (P + P.T)
    w, Z = np.linalg.eigh(P)
    idx = select_ritz_indices(w, which)[:req]
    vals = w[idx]
    C = Z[:, idx]
    X = S[:, :cols] @ C
    AX = AS[:, :cols] @ C
    BX = BS[:, :cols] @ C
    R = AX - BX * vals[None, :]
    rn = np.linalg.norm(R, axis=0)
    bn = np.linalg.norm(BX, axis=0)
    den = (1.0 + np.abs(vals)) * bn
    rel = np.where(den > 0.0, rn / np.where(den > 0.0, den, 1.0), rn)
    if not (np.all(np.isfinite(vals)) and np.all(np.isfinite(rel))):
        raise RuntimeError("non-finite Ritz values or residuals.")
    return vals, C, X, AX, BX, R, rel


def lobpcg_gen_solve(A: Csr, nev: int, B: Optional[Csr] = None, precond: str = "none",
                     block: int = 0, tol: float = 1e-8, maxiter: int = 1000, which: str = "sr",
                     seed: int = 1) -> SolveResult:
    """LOBPCG for K u = l M u (M = I when B is None) with optional Jacobi preconditioning
    and a block of `block` >= nev vectors (convergence on the first nev), loop of
    src/LOBPCGSolver.cpp:25-174 in the B metric; basis [X W P] of at most 3*block columns."""
    n = A.rows
    which = which.lower()
    if n <= 0 or nev <= 0 or nev > n or maxiter <= 0:
        raise ValueError("LOBPCGSolver: require 0 < nev <= n and maxiter > 0.")
    if which not in ("sr", "lr"):
        raise ValueError("LOBPCGSolver: only SR and LR are supported.")
    b = min(n, max(nev, block))
    sign = -1.0 if which == "lr" else 1.0
    Hs = A.scipy()
    H = (lambda X: sign * (Hs @ X))
    t = jacobi_inverse_diagonal(A) if precond == "jacobi" else None
    cap = min(n, 3 * b)
    X0 = random_block(n, b, seed)
    X, BX = ortho_block_b(B, None, None, 0, X0)
    if X is None or X.shape[1] < b:
        raise RuntimeError("LOBPCGSolver: initial block is rank deficient.")
    AX = H(X)
    vals, C, X, AX, BX, R, rel = _gen_ritz(X, AX, BX, b, b, "sr")
    P = None
    it_done = 0
    for it in range(maxiter):
        if rel[:nev].max() <= tol:
            break
        active = [j for j in range(b) if rel[j] > tol]
        Wsrc = R[:, active]
        if t is not None:
            Wsrc = Wsrc * t[:, None]
        X, BX = b_cholesky_qr(B, X)
        S = np.zeros((n, cap))
        BS = np.zeros((n, cap))
        S[:, :b], BS[:, :b] = X, BX
        cols = b
        W, BW = ortho_block_b(B, S, BS, cols, Wsrc)
        if W is not None:
            r = min(W.shape[1], cap - cols)
            S[:, cols:cols + r], BS[:, cols:cols + r] = W[:, :r], BW[:, :r]
            cols += r
        if P is not None and cols < cap:
            Pq, BPq = ortho_block_b(B, S, BS, cols, P[:, active])
            if Pq is not None:
                r = min(Pq.shape[1], cap - cols)
                S[:, cols:cols + r], BS[:, cols:cols + r] = Pq[:, :r], BPq[:, :r]
                cols += r
        AS = H(S[:, :cols])
        vals, C, X, AX, BX, R, rel = _gen_ritz(S, AS, BS, cols, b, "sr")
        Cp = C.copy()
        Cp[:b, :] = 0.0
        P = S[:, :cols] @ Cp
        it_done = it + 1
        if rel[:nev].max() <= tol or cols == b:
            break
    return SolveResult(sign * vals[:nev], X[:, :nev].copy(), rel[:nev].copy(), it_done)


def davidson_gen_solve(A: Csr, nev: int, B: Optional[Csr] = None, precond: str = "none",
                       tol: float = 1e-8, maxiter: int = 1000, which: str = "sr", seed: int = 1,
                       maxblks: int = 10, block: int = 0) -> SolveResult:
    """Block Davidson for K u = l M u with thick restart and optional Jacobi-preconditioned
    corrections (loop of src/DavidsonSolver.cpp:27-264, locktol = min(1e-5, tol), in the
    B metric), on a block of max(nev, block) Ritz vectors (convergence on the first nev)."""
    n = A.rows
    which = which.lower()
    if nev <= 0 or nev > n:
        raise ValueError("DavidsonSolver: nev must be in [1,n].")
    if which not in ("sr", "lr", "sm", "lm", "be"):
        raise ValueError("DavidsonSolver: invalid which option (use SR/LR/SM/LM/BE).")
    Hs = A.scipy()
    H = (lambda X: Hs @ X)
    t = jacobi_inverse_diagonal(A) if precond == "jacobi" else None
    b = min(n, max(nev, block))
    cap = min(n, maxblks * b)
    X0 = random_block(n, b, seed)
    X, BX = ortho_block_b(B, None, None, 0, X0)
    if X is None or X.shape[1] < b:
        raise RuntimeError("DavidsonSolver: initial block is rank deficient.")
    AX = H(X)
    vals, C, X, AX, BX, R, rel = _gen_ritz(X, AX, BX, b, b, which)
    locktol = min(1.0e-5, tol)
    it_done = 0
    for it in range(maxiter):
        X, BX = b_cholesky_qr(B, X)
        V = np.zeros((n, cap))
        BV = np.zeros((n, cap))
        AV = np.zeros((n, cap))
        V[:, :b], BV[:, :b], AV[:, :b] = X, BX, H(X)
        cols = b
        vals, C, X, AX, BX, R, rel = _gen_ritz(V, AV, BV, cols, b, which)
        for _blk in range(1, maxblks):
            active = [j for j in range(b) if rel[j] > locktol]
            cc = len(active)
            if cc == 0 or cols + cc > cap:
                break
            Wsrc = R[:, active]
            if t is not None:
                Wsrc = Wsrc * t[:, None]
            W, BW = ortho_block_b(B, V, BV, cols, Wsrc)
            if W is None:
                break
            r = W.shape[1]
            V[:, cols:cols + r], BV[:, cols:cols + r], AV[:, cols:cols + r] = W, BW, H(W)
            cols += r
            vals, C, X, AX, BX, R, rel = _gen_ritz(V, AV, BV, cols, b, which)
        it_done = it + 1
        if rel[:nev].max() < tol:
            break
    return SolveResult(vals[:nev].copy(), X[:, :nev].copy(), rel[:nev].copy(), it_done)
