"""Row-sharded Chebyshev-filtered subspace iteration over several GPUs.

One process per GPU (``torch.distributed``, NCCL over NVLink for the data path).
The operator's rows are split into contiguous ranges balanced by nonzeros; every
rank owns its rows of the operator and of every block. The only exchanges are
those the algorithm needs:

  * a halo exchange before every SpMM: each rank receives the rows of the block that
    its rows' nonzeros reference on other ranks (point-to-point, ``batch_isend_irecv``;
    for a 1D slab partition of a stencil these are the neighbouring planes);
  * an all-reduce of every FP64 Gram (``X^T Y`` partials, k x m) and of the column
    sums of squares behind norms and residuals.

Everything else is local: the filter steps, rotations and residual blocks run on each
rank's rows, and the small FP64 algebra (Cholesky, triangular inverse, projected
eigenproblem) is replicated from identical all-reduced inputs. The loop is the
reference's ChebyshevSolver::solve (src/ChebyshevSolver.cpp:67-221: Lanczos bounds,
filter, block Gram-Schmidt against locked vectors, Cholesky QR, Rayleigh-Ritz,
ordered locking), with the extensions of the single-GPU solver (``block``,
``bounds="ritz"``, ``locking="hard"``). It starts from the reference's
``std::mt19937`` block (the same global block on every rank count), so a sharded
solve follows the single-process oracle iteration by iteration.

The arithmetic is delegated to a backend. ``CudaShardBackend`` runs this library's
kernels through the C ABI (SpMM on the rank's rectangular local CSR, FP64 Gram and
rotation, device Cholesky, triangular inverse and eigensolver). Tests on the CPU run
the same driver over ``gloo`` with a NumPy backend of the same interface.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

EPS = np.finfo(np.float64).eps


# --------------------------------------------------------------------------
# Partition and halo plan (host logic, no device or communication)
# --------------------------------------------------------------------------


@dataclass
class RankPlan:
    rank: int
    r0: int
    r1: int
    ghosts: np.ndarray                 # global row indices of the ghost rows, sorted
    rowptr: np.ndarray                 # local CSR (rows r0..r1, columns own then ghost)
    colind: np.ndarray
    values: np.ndarray
    sends: dict = field(default_factory=dict)   # peer -> local row indices to send
    recvs: dict = field(default_factory=dict)   # peer -> (first ghost slot, count)

    @property
    def n_own(self) -> int:
        return self.r1 - self.r0

    @property
    def n_ext(self) -> int:
        return self.n_own + self.ghosts.size


def row_bounds(rowptr: np.ndarray, world: int) -> np.ndarray:
    """Contiguous row ranges with about equal nonzeros per rank (world + 1 bounds)."""
    n = rowptr.size - 1
    nnz = int(rowptr[-1])
    targets = (np.arange(1, world) * nnz) // world
    cuts = np.searchsorted(rowptr, targets, side="left")
    bounds = np.concatenate([[0], np.clip(cuts, 0, n), [n]]).astype(np.int64)
    return np.maximum.accumulate(bounds)


def plan_partition(n: int, rowptr, colind, values, world: int) -> list:
    """Per-rank local operators and halo plan of a square CSR split into row ranges."""
    rowptr = np.asarray(rowptr, dtype=np.int64)
    colind = np.asarray(colind, dtype=np.int64)
    values = np.asarray(values, dtype=np.float64)
    bounds = row_bounds(rowptr, world)
    plans = []
    for r in range(world):
        r0, r1 = int(bounds[r]), int(bounds[r + 1])
        s, e = int(rowptr[r0]), int(rowptr[r1])
        cols = colind[s:e]
        outside = (cols < r0) | (cols >= r1)
        ghosts = np.unique(cols[outside])
        local = np.empty(cols.size, dtype=np.int64)
        local[~outside] = cols[~outside] - r0
        local[outside] = (r1 - r0) + np.searchsorted(ghosts, cols[outside])
        plans.append(RankPlan(r, r0, r1, ghosts,
                              (rowptr[r0:r1 + 1] - s).astype(np.int32),
                              local.astype(np.int32), values[s:e].copy()))
    for p in plans:
        owner = np.searchsorted(bounds, p.ghosts, side="right") - 1
        for q in np.unique(owner):
            q = int(q)
            sel = np.flatnonzero(owner == q)
            p.recvs[q] = (int(sel[0]), int(sel.size))  # ghosts are sorted: one run per owner
            plans[q].sends[p.rank] = (p.ghosts[sel] - plans[q].r0).astype(np.int64)
    return plans


# --------------------------------------------------------------------------
# Communication
# --------------------------------------------------------------------------


class Comm:
    """All-reduce and halo exchange over a torch.distributed group."""

    def __init__(self, plan: RankPlan, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.plan = plan
        self.group = group

    def allreduce(self, t):
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
        return t

    def halo(self, X_ext, cols: int):
        """Fill the ghost rows of X_ext[:, :cols] from their owners."""
        import torch
        p = self.plan
        if not p.sends and not p.recvs:
            return
        ops, recv_bufs = [], []
        keep = []
        for q, idx in sorted(p.sends.items()):
            index = torch.as_tensor(idx, device=X_ext.device)
            buf = X_ext[:, :cols].index_select(0, index).contiguous()
            keep.append(buf)
            ops.append(self.dist.P2POp(self.dist.isend, buf, q, group=self.group))
        for q, (first, count) in sorted(p.recvs.items()):
            buf = torch.empty((count, cols), dtype=X_ext.dtype, device=X_ext.device)
            recv_bufs.append((first, count, buf))
            ops.append(self.dist.P2POp(self.dist.irecv, buf, q, group=self.group))
        for req in self.dist.batch_isend_irecv(ops):
            req.wait()
        n_own = p.n_own
        for first, count, buf in recv_bufs:
            X_ext[n_own + first:n_own + first + count, :cols] = buf


# --------------------------------------------------------------------------
# Backend: this library's CUDA kernels
# --------------------------------------------------------------------------


class CudaShardBackend:
    """Device arithmetic of one rank through the C ABI (no CPU fallback: importing
    the library raises if the CUDA build is missing)."""

    def __init__(self, device=None):
        import torch

        from . import ops
        from ._lib import check, lib
        self.torch, self.ops, self.lib, self.check = torch, ops, lib, check
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None \
            else torch.device(device)

    def operator(self, plan: RankPlan):
        from .problem import CsrMatrix
        return CsrMatrix(plan.n_own, plan.rowptr, plan.colind, plan.values, cols=plan.n_ext)

    def block(self, rows: int, cols: int, ld: Optional[int] = None):
        ld = ld or max(8, (cols + 7) // 8 * 8)
        return self.torch.zeros((rows, ld), dtype=self.torch.float64, device=self.device)[:, :cols]

    def from_host(self, a):
        return self.torch.from_numpy(np.ascontiguousarray(a)).to(self.device)

    def to_host(self, t):
        return t.detach().cpu().numpy()

    def spmm(self, A, X_ext, Y, alpha: float):
        self.ops.spmm(A, X_ext, Y, alpha, 0.0)

    def cheb_step(self, A, cur_ext, prev, out, alpha, gamma, beta):
        """out = alpha A cur_ext + gamma cur_own + beta prev (out may be prev); A is the
        rank's rectangular CSR, whose own columns come first."""
        if beta == 0.0 or prev is None:
            prev = out
        ld = cur_ext.stride(0)
        if prev.stride(0) != ld or out.stride(0) != ld:
            raise ValueError("blocks of a filter step must share a leading dimension")
        self.check(self.lib.fe_cheb_step_f64(A.handle, cur_ext.data_ptr(), prev.data_ptr(),
                                             out.data_ptr(), ld, out.shape[1], float(alpha),
                                             float(gamma), float(beta),
                                             self.torch.cuda.current_stream().cuda_stream))

    def gram(self, X, Y):
        return self.ops.gram(X, Y)

    def rotate(self, X, C, Y, alpha=1.0, beta=0.0):
        self.ops.rotate(X, self.from_host(C) if isinstance(C, np.ndarray) else C, Y, alpha, beta)

    def colsq(self, X):
        return self.ops.column_norms(X) ** 2

    def residual_sq(self, AX, X, lam):
        rn, xn, _ = self.ops.residual_norms(AX, X, self.from_host(lam))
        return rn ** 2, xn ** 2

    def cholesky_upper(self, G):
        R, info = self.ops.potrf_upper(self.from_host(G))
        if int(info.item()) != 0:
            return None
        return self.to_host(R)

    def inv_upper(self, R):
        return self.to_host(self.ops.trinv_upper(self.from_host(R)))

    def eigh(self, P):
        k = P.shape[0]
        A = self.from_host(np.asfortranarray(P).T.copy())  # column-major storage
        W = self.torch.zeros(k, dtype=self.torch.float64, device=self.device)
        info = self.torch.zeros(1, dtype=self.torch.int32, device=self.device)
        need = self.lib.fe_syevd_f64_workspace_bytes(k)
        ws = self.torch.empty(max(need, 8), dtype=self.torch.uint8, device=self.device)
        self.check(self.lib.fe_syevd_f64(A.data_ptr(), k, k, W.data_ptr(), info.data_ptr(),
                                         ws.data_ptr(), need,
                                         self.torch.cuda.current_stream().cuda_stream))
        if int(info.item()) != 0:
            raise RuntimeError("ChebyshevSolver: non-finite Ritz values or residuals.")
        return self.to_host(W), self.to_host(A).T.copy()


# --------------------------------------------------------------------------
# The solver
# --------------------------------------------------------------------------


@dataclass
class ShardedResult:
    eigenvalues: np.ndarray
    residual_norms: np.ndarray
    iterations: int
    vectors: object  # the rank's rows of the eigenvectors (backend array)
    r0: int
    r1: int


class _Shard:
    def __init__(self, plan: RankPlan, be, comm: Comm, sign: float):
        self.plan, self.be, self.comm, self.sign = plan, be, comm, sign
        self.A = be.operator(plan)

    def reduce(self, local):
        """All-reduce a small backend array (sum over ranks); returns a host array."""
        return self.be.to_host(self.comm.allreduce(local))

    def gram(self, X, Y):
        return self.reduce(self.be.gram(X, Y).contiguous())

    def apply(self, X, out, ext):
        """out = op X (op = sign A), through the halo of ext (n_ext x >= cols)."""
        cols = X.shape[1]
        ext[:self.plan.n_own, :cols] = X
        self.comm.halo(ext, cols)
        self.be.spmm(self.A, ext[:, :cols], out, self.sign)

    def norms(self, X):
        return np.sqrt(self.reduce(self.be.colsq(X).contiguous()))


def _lanczos_bounds(sh: _Shard, n: int, seed: int, global_vector):
    """estimate_bounds_with_executor (src/ChebyshevSolver.cpp:26-49) over the shards:
    20 Lanczos steps with two-pass classical Gram-Schmidt (src/core/KrylovSubspace.cpp:
    125-259), inner products all-reduced."""
    be, p = sh.be, sh.plan
    steps = min(20, n)
    V = be.block(p.n_own, steps)
    ext = be.block(p.n_ext, 1)
    w = be.block(p.n_own, 1)
    f = be.block(p.n_own, 1)
    f[:, 0] = be.from_host(global_vector(n, seed)[p.r0:p.r1])
    T = np.zeros((steps, steps))
    beta_next = 0.0

    def orthogonalize(k, src):
        r = be.block(p.n_own, 1)
        r[:] = src
        if k == 0:
            return r, 0.0
        h = sh.gram(V[:, :k], r)
        be.rotate(V[:, :k], h, r, -1.0, 1.0)
        s2 = sh.gram(V[:, :k], r)
        be.rotate(V[:, :k], s2, r, -1.0, 1.0)
        return r, float(h[k - 1, 0] + s2[k - 1, 0])

    for it in range(steps):
        beta = float(sh.norms(f)[0])
        restarted = False
        if not math.isfinite(beta):
            raise RuntimeError("non-finite residual norm encountered.")
        if beta <= EPS:
            cand = be.block(p.n_own, 1)
            cand[:, 0] = be.from_host(global_vector(n, seed + it + 1)[p.r0:p.r1])
            f, _ = orthogonalize(it, cand)
            restarted = True
            beta = float(sh.norms(f)[0])
            if beta <= EPS:
                raise RuntimeError("breakdown, unable to generate new basis vector.")
        V[:, it] = f[:, 0] / beta
        sh.apply(V[:, it:it + 1], w, ext)
        f, alpha = orthogonalize(it + 1, w)
        beta_next = float(sh.norms(f)[0])
        if it != 0 and not restarted:
            T[it, it - 1] = T[it - 1, it] = beta
        T[it, it] = alpha
    lam, Z = sh.be.eigh(T)
    rel = np.abs(beta_next * Z[steps - 1, :]) / (1.0 + np.abs(lam))
    r = rel * (1.0 + np.abs(lam))
    lower, upper = float((lam - r).min()), float((lam + r).max())
    if not (math.isfinite(lower) and math.isfinite(upper)) or lower > upper:
        raise RuntimeError("ChebyshevSolver: invalid spectral bound estimates.")
    return lower, upper


def _cholesky_qr(sh: _Shard, X, out):
    """cholesky_qr (src/core/Orthogonalization.cpp:49-57): out = X R^{-1}, G = X^T X."""
    G = sh.gram(X, X)
    R = sh.be.cholesky_upper(G)
    if R is None:
        return False
    sh.be.rotate(X, sh.be.inv_upper(R), out)
    return True


def sharded_chebyshev_solve(n: int, rowptr, colind, values, nev: int, *, degree: int = 10,
                            tol: float = 1e-8, maxiter: int = 1000, which: str = "sr",
                            seed: int = 1, block: Optional[int] = None,
                            bounds: str = "reference", amplification: float = math.inf,
                            locking: str = "soft", rank: int = 0, world: int = 1, group=None,
                            backend=None) -> ShardedResult:
    """ChebyshevSolver::solve on `world` ranks; every rank passes the same global CSR
    (full symmetric storage) and options and gets its rows of the eigenvectors."""
    from .rng import random_block_rows, random_vector
    which = which.lower()
    if n <= 0 or nev <= 0 or nev > n:
        raise ValueError("ChebyshevSolver: nev must be in [1,n].")
    if which not in ("sr", "lr"):
        raise ValueError("ChebyshevSolver: only SR and LR are supported.")
    sign = -1.0 if which == "lr" else 1.0
    plan = plan_partition(n, rowptr, colind, values, world)[rank]
    be = backend if backend is not None else CudaShardBackend()
    sh = _Shard(plan, be, Comm(plan, group), sign)
    no = plan.n_own
    capacity = nev + min(nev, n - nev) if block is None else max(nev, min(block, n))

    # Initial block and its Cholesky QR (src/ChebyshevSolver.cpp:94-107).
    V = be.block(no, capacity)
    start = be.block(no, capacity)
    start[:] = be.from_host(random_block_rows(n, capacity, seed, plan.r0, plan.r1))
    if not _cholesky_qr(sh, start, V):
        raise RuntimeError("ChebyshevSolver: initial Cholesky QR failed.")
    lower, upper = _lanczos_bounds(sh, n, seed, random_vector)

    ext_a = be.block(plan.n_ext, capacity)
    ext_b = be.block(plan.n_ext, capacity)
    Q = be.block(no, capacity)
    AQ = be.block(no, capacity)
    Xr = be.block(no, capacity)
    tmp = be.block(no, capacity)

    def filt(cols, lo_or_cutoff, window):
        # Y0 = X, Y1 = (c op + d) X, Yk = 2 (c op + d) Y_{k-1} - Y_{k-2}
        # (src/ChebyshevSolver.cpp:223-258) on V[:, locked:locked+cols] in place.
        if window:
            cutoff = lo_or_cutoff
            if upper <= cutoff:
                return
        else:
            xlb = math.cosh(math.acosh(1.0e3) / degree)
            if upper == lo_or_cutoff:
                return
            cutoff = (2.0 * lo_or_cutoff + upper * (xlb - 1.0)) / (1.0 + xlb)
        c = 2.0 / (upper - cutoff)
        d = -(upper + cutoff) / (upper - cutoff)
        if not (math.isfinite(c) and math.isfinite(d)):
            raise RuntimeError("ChebyshevSolver: invalid filter scaling.")
        X = V[:, locked:locked + cols]
        prev, cur = ext_a, ext_b
        prev[:no, :cols] = X
        sh.comm.halo(prev, cols)
        be.cheb_step(sh.A, prev[:, :cols], None, cur[:no, :cols], sign * c, d, 0.0)
        for _ in range(2, degree + 1):
            sh.comm.halo(cur, cols)
            be.cheb_step(sh.A, cur[:, :cols], prev[:no, :cols], prev[:no, :cols], 2.0 * sign * c,
                         2.0 * d, -1.0)
            prev, cur = cur, prev
        X[:] = cur[:no, :cols]

    def rayleigh_ritz(basis, cols):
        """extract_projected_ritz_pairs (src/core/RitzExtraction.cpp:65-141) on a
        sharded orthonormal basis: Ritz vectors into Xr[:, :cols]."""
        sh.apply(basis, AQ[:, :cols], ext_a)
        P = sh.gram(basis, AQ[:, :cols])
        P = 0.5 * (P + P.T)
        w, Z = be.eigh(P)
        be.rotate(basis, Z, Xr[:, :cols])
        be.rotate(AQ[:, :cols], Z, tmp[:, :cols])
        rn2, xn2 = be.residual_sq(tmp[:, :cols], Xr[:, :cols], w)
        rn = np.sqrt(sh.reduce(rn2.contiguous()))
        xn = np.sqrt(sh.reduce(xn2.contiguous()))
        den = (1.0 + np.abs(w)) * xn
        rel = np.where(den > 0.0, rn / np.where(den > 0.0, den, 1.0), rn)
        if not (np.all(np.isfinite(w)) and np.all(np.isfinite(rel))):
            raise RuntimeError("ChebyshevSolver: non-finite Ritz values or residuals.")
        return w, rel

    locked = 0
    sub = nev
    sub_prev = 0
    vals = np.zeros(capacity)
    rels = np.zeros(capacity)
    have_ritz = False
    it_done = 0
    for it in range(maxiter):
        active = sub - locked
        if bounds == "ritz" and have_ritz:
            cutoff = float(vals[sub_prev - 1] if locking == "soft" else last_max)
            if math.isfinite(amplification):
                xl = math.cosh(math.acosh(amplification) / degree)
                cutoff = min(cutoff, (2.0 * lower + upper * (xl - 1.0)) / (1.0 + xl))
            filt(active, cutoff, True)
        else:
            filt(active, lower, False)
        Y = V[:, locked:locked + active]
        if locked > 0:
            # block_gram_schmidt, two passes (src/core/Orthogonalization.cpp:482-527)
            for _ in range(2):
                H = sh.gram(V[:, :locked], Y)
                be.rotate(V[:, :locked], H, Y, -1.0, 1.0)
        if locking == "hard":
            if not _cholesky_qr(sh, Y, Q[:, :active]):
                raise RuntimeError("ChebyshevSolver: Cholesky QR failed during filtering.")
            w, rel = rayleigh_ritz(Q[:, :active], active)
            vals[locked:sub] = w
            rels[locked:sub] = rel
            last_max = float(w[-1])
            V[:, locked:sub] = Xr[:, :active]
            sub_prev = sub
            while locked < nev and rels[locked] <= tol:
                locked += 1
        else:
            if not _cholesky_qr(sh, V[:, :sub], Q[:, :sub]):
                raise RuntimeError("ChebyshevSolver: Cholesky QR failed during filtering.")
            w, rel = rayleigh_ritz(Q[:, :sub], sub)
            vals[:sub] = w
            rels[:sub] = rel
            V[:, :sub] = Xr[:, :sub]
            sub_prev = sub
            locked = 0
            while locked < nev and rels[locked] <= tol:
                locked += 1
        have_ritz = True
        sub = max(sub, nev + min(locked, capacity - nev))
        it_done = it + 1
        if rels[:nev].max() <= tol:
            break
    order = np.argsort(vals[:nev], kind="stable") if locking == "hard" else np.arange(nev)
    out = be.block(no, nev)
    for j, o in enumerate(order):
        out[:, j] = V[:, int(o)]
    return ShardedResult(sign * vals[:nev][order], rels[:nev][order].copy(), it_done, out,
                         plan.r0, plan.r1)
