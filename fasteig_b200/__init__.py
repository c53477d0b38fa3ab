"""fasteig_b200: B200-native (sm_100a) backend for fasteig's sparse symmetric
eigensolver hot path (block SpMM, fused Chebyshev filter, CholQR and
Rayleigh-Ritz block kernels) behind fasteig's problem/options API.

The CUDA library is loaded on first use of any public name; if it has not been
built, that access raises ImportError. There is no CPU execution path.
(``fasteig_b200.build`` and ``fasteig_b200.matrices`` import without it.)
"""
import importlib

_LAZY = {
    "FastEigError": "._lib",
    "lib": "._lib",
    "version": "._lib",
    "CsrMatrix": ".problem",
    "fasteig_options": ".problem",
    "fasteig_problem": ".problem",
    "batch_krylov_schur": ".problem",
    "grouped_chebyshev": ".problem",
    "Server": ".problem",
}

__all__ = sorted(_LAZY)


def __getattr__(name):
    mod = _LAZY.get(name)
    if mod is None:
        raise AttributeError(f"module 'fasteig_b200' has no attribute {name!r}")
    value = getattr(importlib.import_module(mod, __name__), name)
    globals()[name] = value
    return value
