"""ctypes binding of the C ABI declared in include/fasteig_b200.h.

The shared library is built in-tree (``python -m fasteig_b200.build``). There is
no fallback: if the library is missing or cannot be loaded, importing this
module raises, so no caller can silently run without the CUDA backend.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libfasteig_b200.so"

if not LIB_PATH.exists():
    raise ImportError(f"fasteig_b200: CUDA library not built ({LIB_PATH}); "
                      "run `python -m fasteig_b200.build`")

lib = C.CDLL(str(LIB_PATH))

i32, i64, f64, vp, sz = C.c_int32, C.c_int64, C.c_double, C.c_void_p, C.c_size_t
P32 = C.POINTER(C.c_int32)
PD = C.POINTER(C.c_double)

_SIGS = {
    "fe_version": (C.c_char_p, []),
    "fe_last_error": (C.c_char_p, []),
    "fe_device_count": (C.c_int, [C.POINTER(C.c_int)]),
    "fe_launch_count": (C.c_int64, []),
    "fe_csr_create": (C.c_int, [i64, i64, i64, vp, vp, vp, C.POINTER(vp)]),
    "fe_csr_destroy": (C.c_int, [vp]),
    "fe_csr_create_from_triplets": (C.c_int, [i64, i64, vp, vp, vp, i32, C.POINTER(vp)]),
    "fe_csr_create_from_matrix_market": (C.c_int, [C.c_char_p, C.POINTER(vp)]),
    "fe_csr_info": (C.c_int, [vp, C.POINTER(i64), C.POINTER(i64), C.POINTER(i64)]),
    "fe_csr_copy_to_host": (C.c_int, [vp, vp, vp, vp]),
    "fe_spmm_csr_f64": (C.c_int, [vp, vp, i64, vp, i64, i64, f64, f64, vp]),
    "fe_spmm_csr_f32": (C.c_int, [vp, vp, i64, vp, i64, i64, f64, f64, vp]),
    "fe_cheb_step_f64": (C.c_int, [vp, vp, vp, vp, i64, i64, f64, f64, f64, vp]),
    "fe_cheb_step_f32": (C.c_int, [vp, vp, vp, vp, i64, i64, f64, f64, f64, vp]),
    "fe_cheb_filter_f64": (C.c_int, [vp, vp, vp, i64, i64, i32, f64, f64, vp]),
    "fe_cheb_filter_f32": (C.c_int, [vp, vp, vp, i64, i64, i32, f64, f64, vp]),
    "fe_gram_workspace_bytes": (sz, [i64, i64, i64]),
    "fe_syevd_f64_workspace_bytes": (sz, [i64]),
    "fe_syevd_f64": (C.c_int, [vp, i64, i64, vp, vp, vp, sz, vp]),
    "fe_selftest_wait_timeout": (C.c_int, [i64, i32, vp]),
    "fe_lanczos_workspace_bytes": (sz, [i64, i64]),
    "fe_lanczos_step": (C.c_int, [vp, vp, i64, i64, i64, vp, vp, vp, i64, vp, sz, vp]),
    "fe_gram_f64": (C.c_int, [vp, i64, vp, i64, i64, i64, i64, vp, i64, vp, sz, vp]),
    "fe_gram_f32": (C.c_int, [vp, i64, vp, i64, i64, i64, i64, vp, i64, vp, sz, vp]),
    "fe_rotate_f64": (C.c_int, [vp, i64, vp, i64, vp, i64, i64, i64, i64, f64, f64, vp]),
    "fe_rotate_f32": (C.c_int, [vp, i64, vp, i64, vp, i64, i64, i64, i64, f64, f64, vp]),
    "fe_residual_workspace_bytes": (sz, [i64, i64]),
    "fe_residual_norms_f64": (C.c_int, [vp, vp, vp, i64, i64, i64, vp, vp, i64, vp, vp, vp, vp,
                                        sz, vp]),
    "fe_residual_norms_f32": (C.c_int, [vp, vp, vp, i64, i64, i64, vp, vp, i64, vp, vp, vp, vp,
                                        sz, vp]),
    "fe_column_norms_f64": (C.c_int, [vp, i64, i64, i64, vp, vp, sz, vp]),
    "fe_column_norms_f32": (C.c_int, [vp, i64, i64, i64, vp, vp, sz, vp]),
    "fe_potrf_upper_f64": (C.c_int, [vp, i64, i64, vp, vp]),
    "fe_trinv_upper_f64": (C.c_int, [vp, i64, vp, i64, i64, vp]),
    "fe_chol_inv_upper_batched_f64": (C.c_int, [C.c_int32, vp, i64, i64, vp, i64, vp, vp]),
    "fe_symmetrize_f64": (C.c_int, [vp, i64, i64, vp]),
    "fe_convert_f64_to_f32": (C.c_int, [vp, i64, vp, i64, i64, i64, vp]),
    "fe_convert_f32_to_f64": (C.c_int, [vp, i64, vp, i64, i64, i64, vp]),
    "fe_solve": (C.c_int, [vp, vp, C.c_char_p, vp, vp, vp, vp]),
    "fe_gram_tf32x3_workspace_bytes": (sz, [i64, i64, i64]),
    "fe_gram_tf32x3": (C.c_int, [vp, i64, vp, i64, i64, i64, i64, vp, i64, vp, sz, vp]),
    "fe_rotate_tf32x3_workspace_bytes": (sz, [i64, i64]),
    "fe_rotate_tf32x3": (C.c_int, [vp, i64, vp, i64, vp, i64, i64, i64, i64, f64, f64, vp, sz,
                                   vp]),
    "fe_device_status": (C.c_int, [C.POINTER(C.c_int32), C.c_int32]),
    "fe_set_spmm_kernel": (C.c_int, [C.c_int32]),
    "fe_set_cheb_wave_kernel": (C.c_int, [C.c_int32]),
    "fe_set_f64_gemm_kernel": (C.c_int, [C.c_int32]),
    "fe_set_tc_rotate_kernel": (C.c_int, [C.c_int32]),
    "fe_set_syevd_kernel": (C.c_int, [C.c_int32]),
    "fe_csr_autotune": (C.c_int, [vp, i64, C.c_int32, vp, vp]),
    "fe_batch_krylov_schur": (C.c_int, [C.c_int32, vp, vp, C.c_char_p, vp, vp, vp, vp, vp, vp]),
    "fe_csr_block_diag": (C.c_int, [C.c_int32, vp, vp]),
    "fe_grouped_chebyshev": (C.c_int, [C.c_int32, vp, vp, vp, vp, vp, vp]),
    "fe_syevd_batched_f64": (C.c_int, [C.c_int32, vp, vp, i64, vp, vp, vp]),
    "fe_server_create": (C.c_int, [C.c_int32, C.c_int32, i64, vp]),
    "fe_server_submit": (C.c_int, [vp, vp, vp, C.c_char_p, vp]),
    "fe_server_wait": (C.c_int, [vp, i64, C.c_double, vp, vp, vp]),
    "fe_server_destroy": (C.c_int, [vp]),
    "fe_server_stats": (C.c_int, [vp, vp, C.c_int32]),
    "fe_gram_f64_noalloc": (C.c_int, [vp, i64, vp, i64, i64, i64, i64, vp, i64, vp]),
    "fe_gram_f64_noalloc_max_entries": (C.c_int64, []),
}

for _name, (_res, _args) in _SIGS.items():
    _fn = getattr(lib, _name)
    _fn.restype = _res
    _fn.argtypes = _args

EXPORTED = tuple(_SIGS)


class FastEigError(RuntimeError):
    """A fasteig_b200 C ABI call returned a non-zero status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code


def check(status: int) -> None:
    if status != 0:
        raise FastEigError(status, lib.fe_last_error().decode(errors="replace"))


def version() -> str:
    return lib.fe_version().decode()
