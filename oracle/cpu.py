"""Threaded host operator for timing the oracle's Chebyshev loop at full size.

TEST INFRASTRUCTURE ONLY (bench.py's CPU legs and tests/). ``ThreadedChebyshevOps``
has the interface of ``oracle.NumpyChebyshevOps`` and the reference CPU backend's
arithmetic (oracle/cpu_kernels.c): each filter step is one row-parallel pass,
``Y = (2c a) X + 2d X - Y_prev`` in place over the k-2 block, as
ChebyshevSolver::chebyshev_filter (src/ChebyshevSolver.cpp:243-256) computes with
copy_from + apply_block(2c, -1) + add_scaled_columns(2d). SciPy's CSR product is
single-threaded and NumPy's elementwise passes are too, so at n = 2M x 320 the
NumPy path takes about ten times longer per filter step than the host's cores allow.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_bin" / "libfe_oracle_cpu.so"
_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB.exists() or LIB.stat().st_mtime < (HERE / "cpu_kernels.c").stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True, capture_output=True)
    lib = C.CDLL(str(LIB))
    i64, f64, ptr = C.c_int64, C.c_double, C.c_void_p
    lib.fe_oracle_csr_step.argtypes = [i64, ptr, ptr, ptr, ptr, i64, ptr, i64, ptr, i64, i64,
                                       f64, f64, f64, C.c_int]
    lib.fe_oracle_csr_step.restype = None
    lib.fe_oracle_residual_norms.argtypes = [i64, i64, ptr, i64, ptr, i64, ptr, ptr, ptr, C.c_int]
    lib.fe_oracle_residual_norms.restype = None
    _lib = lib
    return lib


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def _rowmajor(X):
    if X.ndim == 1:
        return X.reshape(-1, 1), 1
    if X.strides[1] != X.itemsize or X.strides[0] % X.itemsize:
        raise ValueError("row-major block expected")
    return X, X.strides[0] // X.itemsize


class ThreadedChebyshevOps:
    def __init__(self, A, sign: float, threads: int = 0):
        self.lib = load()
        self.n = A.rows
        self.rowptr = np.ascontiguousarray(A.rowptr, dtype=np.int32)
        self.colind = np.ascontiguousarray(A.colind, dtype=np.int32)
        self.values = np.ascontiguousarray(A.values, dtype=np.float64)
        self.sign = sign
        self.threads = threads or host_threads()

    def step(self, cur, prev, out, alpha, gamma, beta):
        """out = alpha*A*cur + beta*prev + gamma*cur (out may be prev)."""
        cur2, ldc = _rowmajor(cur)
        out2, ldo = _rowmajor(out)
        if prev is None:
            pp, ldp = None, 0
        else:
            prev2, ldp = _rowmajor(prev)
            pp = prev2.ctypes.data
        self.lib.fe_oracle_csr_step(self.n, self.rowptr.ctypes.data, self.colind.ctypes.data,
                                    self.values.ctypes.data, cur2.ctypes.data, ldc, pp, ldp,
                                    out2.ctypes.data, ldo, cur2.shape[1], float(alpha),
                                    float(gamma), float(beta), self.threads)

    def apply(self, X):
        X = np.ascontiguousarray(X)
        Y = np.empty_like(X)
        self.step(X, None, Y, self.sign, 0.0, 0.0)
        return Y

    def _recurrence(self, X, degree, c, d):
        X = np.ascontiguousarray(X)
        prev = X
        cur = np.empty_like(X)
        self.step(X, None, cur, self.sign * c, d, 0.0)
        for _ in range(2, degree + 1):
            self.step(cur, prev, prev, 2.0 * self.sign * c, 2.0 * d, -1.0)
            prev, cur = cur, prev
        return cur

    def filter(self, X, degree, lower, upper):
        from .oracle import chebyshev_filter_coefficients
        cd = chebyshev_filter_coefficients(lower, upper, degree)
        if cd is None:
            return X
        return self._recurrence(X, degree, cd[0], cd[1])

    def filter_window(self, X, degree, cutoff, upper):
        if upper <= cutoff:
            return X
        c = 2.0 / (upper - cutoff)
        d = -(upper + cutoff) / (upper - cutoff)
        return self._recurrence(X, degree, c, d)

    def residual_norms(self, AX, X, lam):
        AX2, lda = _rowmajor(AX)
        X2, ldx = _rowmajor(X)
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        k = X2.shape[1]
        rn, xn = np.zeros(k), np.zeros(k)
        self.lib.fe_oracle_residual_norms(self.n, k, AX2.ctypes.data, lda, X2.ctypes.data, ldx,
                                          lam.ctypes.data, rn.ctypes.data, xn.ctypes.data,
                                          self.threads)
        return rn, xn
