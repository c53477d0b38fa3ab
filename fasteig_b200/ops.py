"""Kernel-level entry points on torch CUDA tensors (row-major blocks).

Thin wrappers that pass tensor data pointers, leading dimensions and the
current CUDA stream to the C ABI. Blocks are 2-D row-major tensors (stride(1)
must be 1); small matrices (Gram, coefficients) are FP64 column-major, which
for a torch tensor means a (k, m) tensor viewed through ``.T`` of a contiguous
(m, k) tensor; ``gram`` and friends handle that layout for the caller.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

import torch

from ._lib import check, lib
from .problem import CsrMatrix


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def _rowmajor(t: torch.Tensor, name: str) -> int:
    if t.dim() != 2 or t.stride(1) != 1:
        raise ValueError(f"{name} must be a 2-D row-major tensor")
    return t.stride(0)


def _fn(base: str, t: torch.Tensor):
    if t.dtype == torch.float64:
        return getattr(lib, base + "_f64")
    if t.dtype == torch.float32:
        return getattr(lib, base + "_f32")
    raise TypeError(f"unsupported dtype {t.dtype}")


def spmm(A: CsrMatrix, X: torch.Tensor, Y: torch.Tensor, alpha: float = 1.0, beta: float = 0.0):
    """Y[:, :b] = alpha*A*X + beta*Y (b = X.shape[1])."""
    ldx, ldy = _rowmajor(X, "X"), _rowmajor(Y, "Y")
    check(_fn("fe_spmm_csr", X)(A.handle, X.data_ptr(), ldx, Y.data_ptr(), ldy, X.shape[1],
                                float(alpha), float(beta), _stream()))
    return Y


def cheb_step(A: CsrMatrix, Ycur: torch.Tensor, Yprev: torch.Tensor, Yout: torch.Tensor,
              alpha: float, gamma: float, beta: float):
    """Yout = alpha*A*Ycur + gamma*Ycur + beta*Yprev (Yout may alias Yprev)."""
    ld = _rowmajor(Ycur, "Ycur")
    if Yprev.stride(0) != ld or Yout.stride(0) != ld:
        raise ValueError("cheb_step blocks must share a leading dimension")
    check(_fn("fe_cheb_step", Ycur)(A.handle, Ycur.data_ptr(), Yprev.data_ptr(), Yout.data_ptr(),
                                    ld, Ycur.shape[1], float(alpha), float(gamma), float(beta),
                                    _stream()))
    return Yout


def cheb_filter(A: CsrMatrix, X: torch.Tensor, scratch: torch.Tensor, degree: int, c: float,
                d: float):
    ld = _rowmajor(X, "X")
    if scratch.stride(0) != ld:
        raise ValueError("scratch must share X's leading dimension")
    check(_fn("fe_cheb_filter", X)(A.handle, X.data_ptr(), scratch.data_ptr(), ld, X.shape[1],
                                   int(degree), float(c), float(d), _stream()))
    return X


def gram(X: torch.Tensor, Y: torch.Tensor, workspace: torch.Tensor = None) -> torch.Tensor:
    """G = X^T Y as an FP64 (k, m) tensor (stored column-major on the device)."""
    ldx, ldy = _rowmajor(X, "X"), _rowmajor(Y, "Y")
    n, k = X.shape
    m = Y.shape[1]
    Gt = torch.empty((m, k), dtype=torch.float64, device=X.device)  # column-major k x m
    need = lib.fe_gram_workspace_bytes(n, k, m)
    if workspace is None or workspace.numel() * workspace.element_size() < need:
        workspace = torch.empty(max(need, 8), dtype=torch.uint8, device=X.device)
    check(_fn("fe_gram", X)(X.data_ptr(), ldx, Y.data_ptr(), ldy, n, k, m, Gt.data_ptr(), k,
                            workspace.data_ptr(), need, _stream()))
    return Gt.T


def colmajor(Cm: torch.Tensor) -> torch.Tensor:
    """FP64 (k, m) matrix as a column-major device buffer (returns the (m, k) storage)."""
    return Cm.to(torch.float64).T.contiguous()


def rotate(X: torch.Tensor, Cm: torch.Tensor, Y: torch.Tensor, alpha: float = 1.0,
           beta: float = 0.0):
    """Y = alpha*X*C + beta*Y with C an FP64 (k, m) matrix."""
    ldx, ldy = _rowmajor(X, "X"), _rowmajor(Y, "Y")
    n, k = X.shape
    m = Cm.shape[1]
    Cs = colmajor(Cm)
    check(_fn("fe_rotate", X)(X.data_ptr(), ldx, Cs.data_ptr(), k, Y.data_ptr(), ldy, n, k, m,
                              float(alpha), float(beta), _stream()))
    return Y


def residual_norms(AX: torch.Tensor, X: torch.Tensor, lam: torch.Tensor, BX: torch.Tensor = None,
                   R: torch.Tensor = None):
    """R = AX - lam*MX with FP64 norms; returns (rnorm, xnorm, rel)."""
    ld = _rowmajor(X, "X")
    n, m = X.shape
    rn = torch.empty(m, dtype=torch.float64, device=X.device)
    xn = torch.empty_like(rn)
    rel = torch.empty_like(rn)
    need = lib.fe_residual_workspace_bytes(n, m)
    ws = torch.empty(max(need, 8), dtype=torch.uint8, device=X.device)
    lam = lam.to(torch.float64).contiguous()
    check(_fn("fe_residual_norms", X)(AX.data_ptr(), X.data_ptr(),
                                      BX.data_ptr() if BX is not None else None, ld, n, m,
                                      lam.data_ptr(), R.data_ptr() if R is not None else None,
                                      R.stride(0) if R is not None else 0, rn.data_ptr(),
                                      xn.data_ptr(), rel.data_ptr(), ws.data_ptr(), need,
                                      _stream()))
    return rn, xn, rel


def column_norms(X: torch.Tensor) -> torch.Tensor:
    ld = _rowmajor(X, "X")
    n, m = X.shape
    out = torch.empty(m, dtype=torch.float64, device=X.device)
    need = lib.fe_residual_workspace_bytes(n, m)
    ws = torch.empty(max(need, 8), dtype=torch.uint8, device=X.device)
    check(_fn("fe_column_norms", X)(X.data_ptr(), ld, n, m, out.data_ptr(), ws.data_ptr(), need,
                                    _stream()))
    return out


def potrf_upper(G: torch.Tensor):
    """Upper Cholesky of an FP64 (k, k) symmetric matrix; returns (R, info)."""
    k = G.shape[0]
    Gs = colmajor(G)
    info = torch.zeros(1, dtype=torch.int32, device=G.device)
    check(lib.fe_potrf_upper_f64(Gs.data_ptr(), k, k, info.data_ptr(), _stream()))
    return Gs.T, info


def trinv_upper(R: torch.Tensor) -> torch.Tensor:
    k = R.shape[0]
    Rs = colmajor(R)
    out = torch.empty_like(Rs)
    check(lib.fe_trinv_upper_f64(Rs.data_ptr(), k, out.data_ptr(), k, k, _stream()))
    return out.T


def gram_tf32x3(X: torch.Tensor, Y: torch.Tensor) -> torch.Tensor:
    """G = X^T Y on tensor cores (FP32 blocks, 3xTF32 split, FP64 chunk reduction)."""
    ldx, ldy = _rowmajor(X, "X"), _rowmajor(Y, "Y")
    n, k = X.shape
    m = Y.shape[1]
    Gt = torch.empty((m, k), dtype=torch.float64, device=X.device)
    need = lib.fe_gram_tf32x3_workspace_bytes(n, k, m)
    ws = torch.empty(max(need, 8), dtype=torch.uint8, device=X.device)
    check(lib.fe_gram_tf32x3(X.data_ptr(), ldx, Y.data_ptr(), ldy, n, k, m, Gt.data_ptr(), k,
                             ws.data_ptr(), need, _stream()))
    return Gt.T


def rotate_tf32x3(X: torch.Tensor, Cm: torch.Tensor, Y: torch.Tensor, alpha: float = 1.0,
                  beta: float = 0.0):
    """Y = alpha*X*C + beta*Y on tensor cores (FP32 blocks, 3xTF32 split)."""
    ldx, ldy = _rowmajor(X, "X"), _rowmajor(Y, "Y")
    n, k = X.shape
    m = Cm.shape[1]
    Cs = colmajor(Cm)
    need = lib.fe_rotate_tf32x3_workspace_bytes(k, m)
    ws = torch.empty(max(need, 8), dtype=torch.uint8, device=X.device)
    check(lib.fe_rotate_tf32x3(X.data_ptr(), ldx, Cs.data_ptr(), k, Y.data_ptr(), ldy, n, k, m,
                               float(alpha), float(beta), ws.data_ptr(), need, _stream()))
    return Y


def device_status(clear: bool = False) -> int:
    v = C.c_int32()
    check(lib.fe_device_status(C.byref(v), 1 if clear else 0))
    return int(v.value)


def syevd_batched(A: torch.Tensor, sizes) -> tuple:
    """Eigen-decomposition of a batch of small symmetric FP64 matrices
    (``fe_syevd_batched_f64``). A: CUDA float64 (count, lda, lda); matrix p occupies
    its leading sizes[p] x sizes[p] block. Returns (W, Z) with W[p, :m] ascending and
    Z[p, :m, :m] holding the eigenvectors as columns."""
    assert A.is_cuda and A.dtype == torch.float64 and A.dim() == 3 and A.is_contiguous()
    count, lda, _ = A.shape
    m = np.ascontiguousarray(np.asarray(sizes, dtype=np.int32))
    W = torch.zeros((count, lda), dtype=torch.float64, device=A.device)
    Zc = torch.zeros((count, lda, lda), dtype=torch.float64, device=A.device)
    # A is symmetric, so its row-major and column-major storage agree.
    check(lib.fe_syevd_batched_f64(count, m.ctypes.data, A.data_ptr(), lda, W.data_ptr(),
                                   Zc.data_ptr(), _stream()))
    return W, Zc.transpose(1, 2)  # column-major storage -> Z[p][i, j] = component i of vector j
