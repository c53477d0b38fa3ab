"""Dense eigenvalues of the seeded benchmark-shaped matrices, for the GPU parity tests
at the configured sizes.

  * 24^3 7-point Dirichlet Laplacian + U[0,1) diagonal potential (PCG64 seed 0):
    n = 13,824, the LOBPCG configuration (8 lowest pairs, block 12). Lowest 16
    eigenvalues of the dense matrix (LAPACK syevr).
  * 20^3 27-point stiffness / mass pair (log-normal node coefficients, PCG64
    seed 0; M = M1 (x) M1 (x) M1): n = 8,000, the generalized configuration's
    operator family at a size dense LAPACK finishes in seconds. Lowest 96
    generalized eigenvalues of (K, M) (LAPACK sygvd-style reduction).

The dense solves take about a minute on 8 cores, so the values are committed
(tests/golden/dense_spectra.json) instead of recomputed by every test run.
Usage: python tests/golden/make_dense_spectra.py
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import scipy.linalg as sl

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))


def _dense(H):
    import scipy.sparse as sp
    return sp.csr_matrix((H.values, H.colind, H.rowptr), shape=(H.n, H.n)).toarray()


def main():
    from fasteig_b200 import matrices as M
    out = {}
    H = M.laplacian_uniform_potential(24, seed=0)
    w = sl.eigh(_dense(H), eigvals_only=True, subset_by_index=[0, 15], driver="evr")
    out["lobpcg_24cube_uniform_seed0"] = {"n": H.n, "nnz": H.nnz, "lowest": [float(x) for x in w]}
    K, Mm = M.stiffness_mass_27pt(20, seed=0)
    wg = sl.eigh(_dense(K), _dense(Mm), eigvals_only=True, subset_by_index=[0, 95])
    out["generalized_27pt_20cube_seed0"] = {"n": K.n, "nnz_K": K.nnz,
                                            "lowest": [float(x) for x in wg]}
    (HERE / "dense_spectra.json").write_text(json.dumps(out, indent=1))
    print("written", HERE / "dense_spectra.json")


if __name__ == "__main__":
    main()
