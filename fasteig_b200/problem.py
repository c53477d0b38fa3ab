"""Python mirror of fasteig's public problem/options API on the B200 backend.

``fasteig_options`` keeps the reference's key names and defaults
(include/fasteig_options.hpp:102-118, set() keys src/fasteig_options.cpp:51-112);
``fasteig_problem`` keeps ``solve(opts)``, ``eigenvalues()``, ``eigenvectors()``,
``residual_norms()``, ``status()`` and ``last_iterations()``
(include/fasteig_problem.hpp:33-108). Solves run through ``fe_solve`` of the C
ABI; there is no CPU code path.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from ._lib import check, lib

_INT_KEYS = ("n", "nev", "maxiter", "maxdim", "maxblks", "degree", "blksize", "verbosity",
             "print_every", "block", "tensor_cores", "tail_degree", "tail_guard",
             "inject_wait_timeout", "group")
_FLOAT_KEYS = ("tol", "shift", "amplification", "mixed_switch")
_STR_KEYS = ("which", "solver", "precision", "bounds", "init", "logfile", "output_format",
             "precond", "locking", "rr", "tail_filter", "tail_rr")


class fasteig_options:  # noqa: N801 - reference class name
    """Solver configuration (include/fasteig_options.hpp:21-134)."""

    def __init__(self, n: int = 0):
        self._kv = {"n": n, "nev": 10, "maxiter": 1000, "maxdim": 0, "maxblks": 10,
                    "degree": 10, "blksize": 1, "which": "LM", "solver": "Lanczos",
                    "shift": 0.0, "tol": 1.0e-8, "seed": None, "verbosity": 1,
                    "print_every": 0}
        self.v0 = None

    def set(self, key: str, value) -> bool:
        """fasteig_options::set: False for unknown keys, ValueError for bad values."""
        k = key.lower()
        if k == "seed":
            s = int(value)
            if s < 0:
                self._kv["seed"] = None
            elif s > 0xFFFFFFFF:
                raise ValueError("seed out of range for unsigned int")
            else:
                self._kv["seed"] = s
            return True
        if k in _INT_KEYS:
            self._kv[k] = int(value)
        elif k in _FLOAT_KEYS:
            self._kv[k] = float(value)
        elif k in _STR_KEYS:
            self._kv[k] = str(value)
        elif k == "gpu_backend":
            return True  # this backend is always the GPU
        else:
            return False
        return True

    def get(self, key: str):
        k = key.lower()
        if k not in self._kv:
            raise KeyError(key)
        return self._kv[k]

    def validate(self) -> None:
        """fasteig_options::validate essentials."""
        if self._kv["nev"] <= 0:
            raise ValueError("nev must be positive")
        if self._kv["maxiter"] <= 0:
            raise ValueError("maxiter must be positive")
        if not self._kv["tol"] > 0:
            raise ValueError("tol must be positive")

    def nev(self) -> int:
        return int(self._kv["nev"])

    def to_text(self) -> str:
        lines = []
        for k, v in self._kv.items():
            if k in ("n", "verbosity", "print_every", "logfile", "output_format") and k != "verbosity":
                continue
            if v is None:
                continue
            if k == "verbosity" and int(v) < 2:
                continue
            lines.append(f"{k}={v}")
        return "\n".join(lines)


class CsrMatrix:
    """Device CSR operator owned by the backend (CudaCsrMatrix equivalent)."""

    def __init__(self, n: int, rowptr, colind, values, cols: Optional[int] = None):
        self.rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
        self.colind = np.ascontiguousarray(colind, dtype=np.int32)
        self.values = np.ascontiguousarray(values, dtype=np.float64)
        self.rows = int(n)
        self.cols = int(n if cols is None else cols)
        h = C.c_void_p()
        check(lib.fe_csr_create(self.rows, self.cols, int(self.values.size),
                                self.rowptr.ctypes.data, self.colind.ctypes.data,
                                self.values.ctypes.data, C.byref(h)))
        self.handle = h

    @property
    def nnz(self) -> int:
        if self.values is not None:
            return int(self.values.size)
        z = C.c_int64()
        check(lib.fe_csr_info(self.handle, None, None, C.byref(z)))
        return int(z.value)

    @classmethod
    def _from_handle(cls, h) -> "CsrMatrix":
        obj = cls.__new__(cls)
        obj.handle = h
        obj.rowptr = obj.colind = obj.values = None
        r, c = C.c_int64(), C.c_int64()
        check(lib.fe_csr_info(h, C.byref(r), C.byref(c), None))
        obj.rows, obj.cols = int(r.value), int(c.value)
        return obj

    @classmethod
    def from_triplets(cls, n: int, rows, cols, values, expand: str = "none") -> "CsrMatrix":
        """Device CSR built on the GPU from 0-based triplets (``fe_csr_create_from_triplets``):
        duplicates summed in input order, ``expand`` = "none", "symmetric" (one triangle
        given) or "skew", as fasteig_problem::build_sparse_matrix_from_triplets followed by
        build_csr_from_sparse_matrix (src/fasteig_problem.cpp:474-607)."""
        codes = {"none": 0, "symmetric": 1, "skew": 2}
        r = np.ascontiguousarray(rows, dtype=np.int32)
        c = np.ascontiguousarray(cols, dtype=np.int32)
        v = np.ascontiguousarray(values, dtype=np.float64)
        if not (r.size == c.size == v.size):
            raise ValueError("Triplet arrays inconsistent with nnz.")
        h = C.c_void_p()
        check(lib.fe_csr_create_from_triplets(int(n), int(v.size), r.ctypes.data, c.ctypes.data,
                                              v.ctypes.data, codes[expand], C.byref(h)))
        return cls._from_handle(h)

    @classmethod
    def from_matrix_market(cls, path) -> "CsrMatrix":
        """MatrixMarket coordinate file read on the host and built on the GPU
        (``fe_csr_create_from_matrix_market``; symmetric files expand their triangle)."""
        h = C.c_void_p()
        check(lib.fe_csr_create_from_matrix_market(str(path).encode(), C.byref(h)))
        return cls._from_handle(h)

    def to_host(self):
        """(rowptr, colind, values) of the stored matrix (CsrMatrix::copy_to_host)."""
        z = C.c_int64()
        check(lib.fe_csr_info(self.handle, None, None, C.byref(z)))
        rp = np.zeros(self.rows + 1, dtype=np.int32)
        ci = np.zeros(max(int(z.value), 1), dtype=np.int32)
        va = np.zeros(max(int(z.value), 1), dtype=np.float64)
        check(lib.fe_csr_copy_to_host(self.handle, rp.ctypes.data, ci.ctypes.data, va.ctypes.data))
        return rp, ci[:int(z.value)], va[:int(z.value)]

    @classmethod
    def block_diag(cls, parts) -> "CsrMatrix":
        """Block-diagonal operator of device CSR parts (``fe_csr_block_diag``): an SpMM
        on it is the grouped SpMM of all parts."""
        parts = list(parts)
        handles = (C.c_void_p * len(parts))(*[p.handle for p in parts])
        h = C.c_void_p()
        check(lib.fe_csr_block_diag(len(parts), C.cast(handles, C.c_void_p), C.byref(h)))
        obj = cls.__new__(cls)
        obj.handle = h
        obj.rowptr = obj.colind = obj.values = None
        obj.rows = sum(p.rows for p in parts)
        obj.cols = sum(p.cols for p in parts)
        return obj

    def autotune(self, ncols: int, precision: str = "fp32") -> int:
        """Pick the fastest SpMM kernel for n x ncols blocks on this operator
        (``fe_csr_autotune``); returns the chosen kernel mode."""
        mode = C.c_int32()
        check(lib.fe_csr_autotune(self.handle, int(ncols), 1 if precision == "fp32" else 0, None,
                                  C.byref(mode)))
        return int(mode.value)

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib.fe_csr_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class fasteig_problem:  # noqa: N801 - reference class name
    """Standard (A x = l x) or generalized (A x = l B x) sparse symmetric problem."""

    def __init__(self, A: CsrMatrix, B: Optional[CsrMatrix] = None, solver: str = "Lanczos"):
        self.A = A
        self.B = B
        self._solver = solver
        self._eigvals = np.zeros(0)
        self._resnrms = np.zeros(0)
        self._eigvecs = np.zeros((A.rows, 0))
        self._status = 0
        self._iters = None
        self.stats = {}

    def n(self) -> int:
        return self.A.rows

    def is_generalized(self) -> bool:
        return self.B is not None

    def solve(self, opts: Optional[fasteig_options] = None, want_vectors: bool = True,
              vectors_out: Optional[np.ndarray] = None) -> int:
        """Run the solver. ``vectors_out`` (optional) is a caller-owned C-contiguous
        float64 array of shape (nev, n) (column-major n x nev), e.g. a view of pinned
        host memory, that receives the eigenvectors directly."""
        opts = opts or fasteig_options(self.n())
        opts.validate()
        text = opts.to_text()
        if "solver=" not in text:
            text += f"\nsolver={self._solver}"
        nev = opts.nev()
        vals = np.zeros(nev)
        res = np.zeros(nev)
        if vectors_out is not None:
            if (vectors_out.dtype != np.float64 or vectors_out.shape != (nev, self.n())
                    or not vectors_out.flags["C_CONTIGUOUS"]):
                raise ValueError("vectors_out must be a C-contiguous float64 (nev, n) array")
            vecs = vectors_out
        else:
            vecs = np.empty((nev, self.n())) if want_vectors else None  # column-major n x nev
        stats = np.zeros(12)
        check(lib.fe_solve(self.A.handle, self.B.handle if self.B is not None else None,
                           text.encode(), vals.ctypes.data, res.ctypes.data,
                           vecs.ctypes.data if vecs is not None else None, stats.ctypes.data))
        self._eigvals, self._resnrms = vals, res
        self._eigvecs = vecs.T if vecs is not None else None
        self._status = int(stats[1])
        self._iters = int(stats[0])
        self.stats = dict(iterations=int(stats[0]), status=int(stats[1]), seconds=float(stats[2]),
                          spmm_launches=int(stats[3]), fp32_iterations=int(stats[4]),
                          fp64_iterations=int(stats[5]), lower=float(stats[6]),
                          upper=float(stats[7]), filter_ms=float(stats[8]),
                          ortho_ms=float(stats[9]), rr_ms=float(stats[10]),
                          precise_grams=int(stats[11]))
        return self._status

    def eigenvalues(self) -> np.ndarray:
        return self._eigvals

    def eigenvectors(self) -> np.ndarray:
        return self._eigvecs

    def residual_norms(self) -> np.ndarray:
        return self._resnrms

    def status(self) -> int:
        return self._status

    def last_iterations(self):
        return self._iters


def batch_krylov_schur(problems, nevs, opts: Optional[fasteig_options] = None,
                       want_vectors: bool = False):
    """Solve many independent standard problems together with the batched
    Krylov-Schur engine (``fe_batch_krylov_schur``). ``problems`` are device
    ``CsrMatrix`` objects, ``nevs`` the wanted pair counts. Returns a list of dicts
    (eigenvalues, residual_norms, eigenvectors or None, iterations, status) and the
    batch stats (seconds, rounds, steps, graph_launches)."""
    problems = list(problems)
    nevs = np.ascontiguousarray(np.asarray(nevs, dtype=np.int64))
    if len(problems) != nevs.size or not problems:
        raise ValueError("one nev per problem is required")
    opts = opts or fasteig_options()
    text = opts.to_text()
    count = len(problems)
    handles = (C.c_void_p * count)(*[p.handle for p in problems])
    total = int(nevs.sum())
    vals = np.zeros(total)
    res = np.zeros(total)
    sizes = [p.rows * int(k) for p, k in zip(problems, nevs)]
    vecs = np.zeros(sum(sizes)) if want_vectors else None
    iters = np.zeros(count, dtype=np.int32)
    status = np.zeros(count, dtype=np.int32)
    stats = np.zeros(4)
    check(lib.fe_batch_krylov_schur(count, C.cast(handles, C.c_void_p), nevs.ctypes.data,
                                    text.encode(), vals.ctypes.data, res.ctypes.data,
                                    vecs.ctypes.data if vecs is not None else None,
                                    iters.ctypes.data, status.ctypes.data, stats.ctypes.data))
    out, off, voff = [], 0, 0
    for p, k, sz in zip(problems, nevs, sizes):
        k = int(k)
        ev = None
        if vecs is not None:
            ev = vecs[voff:voff + sz].reshape(k, p.rows).T
            voff += sz
        out.append(dict(eigenvalues=vals[off:off + k], residual_norms=res[off:off + k],
                        eigenvectors=ev))
        off += k
    for d, it, st in zip(out, iters, status):
        d["iterations"] = int(it)
        d["status"] = int(st)
    return out, dict(seconds=float(stats[0]), rounds=int(stats[1]), steps=int(stats[2]),
                     graph_launches=int(stats[3]))


GROUP_STATS = 11


def grouped_chebyshev(problems, opts, want_vectors: bool = False):
    """Solve standard problems together with the grouped Chebyshev engine
    (``fe_grouped_chebyshev``): problems of one subspace width and filter degree
    advance as one group, a cycle of grouped kernels (one CUDA graph once the
    membership is stable) per step, and leave as they converge. ``problems`` are
    device ``CsrMatrix`` objects, ``opts`` one ``fasteig_options`` or one per
    problem. Returns a list of dicts (eigenvalues, residual_norms, eigenvectors or
    None, iterations, status, seconds, width, lower, upper) and the batch stats
    (cycles, graph_replays, repacks)."""
    problems = list(problems)
    if not problems:
        raise ValueError("empty batch")
    if isinstance(opts, fasteig_options):
        opts = [opts] * len(problems)
    opts = list(opts)
    if len(opts) != len(problems):
        raise ValueError("one option set per problem is required")
    count = len(problems)
    texts = []
    for o in opts:
        o.validate()
        texts.append(o.to_text().encode())
    handles = (C.c_void_p * count)(*[p.handle for p in problems])
    c_texts = (C.c_char_p * count)(*texts)
    vals = [np.zeros(o.nev()) for o in opts]
    res = [np.zeros(o.nev()) for o in opts]
    vecs = [np.zeros(o.nev() * p.rows) if want_vectors else None for p, o in zip(problems, opts)]
    pv = (C.c_void_p * count)(*[v.ctypes.data for v in vals])
    pr = (C.c_void_p * count)(*[r.ctypes.data for r in res])
    pe = (C.c_void_p * count)(*[v.ctypes.data if v is not None else None for v in vecs])
    stats = np.zeros(count * GROUP_STATS)
    check(lib.fe_grouped_chebyshev(count, C.cast(handles, C.c_void_p), C.cast(c_texts, C.c_void_p),
                                   C.cast(pv, C.c_void_p), C.cast(pr, C.c_void_p),
                                   C.cast(pe, C.c_void_p) if want_vectors else None,
                                   stats.ctypes.data))
    out = []
    for i, (p, o) in enumerate(zip(problems, opts)):
        st = stats[i * GROUP_STATS:(i + 1) * GROUP_STATS]
        ev = vecs[i].reshape(o.nev(), p.rows).T if want_vectors else None
        out.append(dict(eigenvalues=vals[i], residual_norms=res[i], eigenvectors=ev,
                        iterations=int(st[0]), status=int(st[1]), seconds=float(st[2]),
                        width=int(st[3]), lower=float(st[4]), upper=float(st[5]),
                        fp32_iterations=int(st[10])))
    st = stats[:GROUP_STATS]
    return out, dict(cycles=int(st[6]), graph_replays=int(st[7]), repacks=int(st[8]))


class Server:
    """Request server over ``fe_server_*``: requests (operator + options) are
    admitted as worker slots and device memory free up, run concurrently on their
    own streams, and are collected with ``wait``. Chebyshev requests whose options
    set ``group=1`` (FP64 or mixed precision, soft locking) run instead in the grouped
    lane of their subspace width and degree: they join the lane's group between
    filter cycles and advance with the other admitted members in grouped kernels
    (``stats()`` reports the lanes' counters). Keep each request's CsrMatrix alive
    until it is collected."""

    PENDING = 1

    def __init__(self, slots: int = 4, memory_budget_bytes: int = 0, device: int = 0):
        h = C.c_void_p()
        check(lib.fe_server_create(int(device), int(slots), int(memory_budget_bytes), C.byref(h)))
        self.handle = h
        self._nev = {}
        self._keep = {}

    def submit(self, A: CsrMatrix, opts: fasteig_options, B: Optional[CsrMatrix] = None,
               solver: Optional[str] = None) -> int:
        opts.validate()
        text = opts.to_text()
        if solver is not None:
            text += f"\nsolver={solver}"
        rid = C.c_int64()
        check(lib.fe_server_submit(self.handle, A.handle, B.handle if B is not None else None,
                                   text.encode(), C.byref(rid)))
        self._nev[rid.value] = opts.nev()
        self._keep[rid.value] = (A, B)
        return rid.value

    def wait(self, request_id: int, timeout: float = -1.0):
        """Result dict, or None if the request is still pending after ``timeout`` s."""
        nev = self._nev[request_id]
        vals, res, stats = np.zeros(nev), np.zeros(nev), np.zeros(18)
        rc = lib.fe_server_wait(self.handle, int(request_id), float(timeout), vals.ctypes.data,
                                res.ctypes.data, stats.ctypes.data)
        if rc == self.PENDING:
            return None
        self._nev.pop(request_id)
        self._keep.pop(request_id)
        check(rc)
        return dict(eigenvalues=vals, residual_norms=res, iterations=int(stats[0]),
                    status=int(stats[1]), solve_seconds=float(stats[2]),
                    queued_s=float(stats[12]), running_s=float(stats[13]),
                    latency_s=float(stats[14]), admitted_bytes=int(stats[15]),
                    start_s=float(stats[16]), end_s=float(stats[17]))

    def stats(self) -> dict:
        """Counters of the grouped lanes (requests submitted with group=1)."""
        out = np.zeros(6)
        check(lib.fe_server_stats(self.handle, out.ctypes.data, 6))
        keys = ("grouped_served", "group_cycles", "graph_replays", "repacks", "lanes",
                "max_group_members")
        return {k: int(v) for k, v in zip(keys, out)}

    def close(self) -> None:
        if getattr(self, "handle", None):
            check(lib.fe_server_destroy(self.handle))
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
