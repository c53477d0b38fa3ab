"""fasteig_b200: B200-native (sm_100a) backend for fasteig's sparse symmetric
eigensolver hot path (block SpMM, fused Chebyshev filter, CholQR and
Rayleigh-Ritz block kernels) behind fasteig's problem/options API.

Importing the package loads the in-tree CUDA library; it raises ImportError if
the library has not been built. There is no CPU execution path.
"""
from ._lib import FastEigError, lib, version  # noqa: F401
from .problem import CsrMatrix, fasteig_options, fasteig_problem  # noqa: F401

__all__ = ["CsrMatrix", "FastEigError", "fasteig_options", "fasteig_problem", "lib", "version"]
