"""Regenerate the committed golden fixtures from the reference checkout.

Reads (read-only) the reference's own test inputs and known answers:
  examples/Sparse_Matrices/{SiO,Kuu,Muu}.mtx   (symmetric MatrixMarket, lower triangle)
  tests/reference/SiO.out.121mpi               (33,401 ScaLAPACK eigenvalues)
  tests/reference/KuuMuu_eig.txt               (7,102 generalized eigenvalues)
and runs the g++ build of oracle/rng_golden.cpp for std::mt19937 known answers.

Writes tests/golden/{SiO.npz, KuuMuu.npz, spectra.json, mt19937.json}.
Usage: python tests/golden/make_fixtures.py /path/to/fasteig-checkout
"""
from __future__ import annotations

import json
import re
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]


def read_triangle(path: Path):
    with open(path) as f:
        banner = f.readline().lower().split()
        assert banner[0] == "%%matrixmarket" and banner[2] == "coordinate", banner
        line = f.readline()
        while line.startswith("%"):
            line = f.readline()
        n, _, nz = (int(t) for t in line.split())
        data = np.loadtxt(f, dtype=np.float64, ndmin=2, max_rows=nz)
    assert data.shape[0] == nz, (path, data.shape, nz)
    return n, banner[4], (data[:, 0] - 1).astype(np.int32), (data[:, 1] - 1).astype(np.int32), data[:, 2]


def spectrum(path: Path):
    txt = path.read_text()
    vals = {int(m.group(1)): float(m.group(2).replace("D", "E").replace("d", "e"))
            for m in re.finditer(r"ev\(\s*(\d+)\s*\)\s*=\s*([+-]?[\d.]+(?:[eEdD][+-]?\d+)?)", txt)}
    return [vals[i] for i in range(1, len(vals) + 1)]


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_fixtures.py /path/to/fasteig-checkout")
    REF = Path(sys.argv[1])
    mats = REF / "examples" / "Sparse_Matrices"
    n, sym, r, c, v = read_triangle(mats / "SiO.mtx")
    np.savez_compressed(HERE / "SiO.npz", n=n, symmetric=sym == "symmetric", row=r, col=c, val=v)
    nk, symk, rk, ck, vk = read_triangle(mats / "Kuu.mtx")
    nm, symm, rm, cm, vm = read_triangle(mats / "Muu.mtx")
    np.savez_compressed(HERE / "KuuMuu.npz", n=nk, k_row=rk, k_col=ck, k_val=vk,
                        m_row=rm, m_col=cm, m_val=vm)
    sio = sorted(spectrum(REF / "tests" / "reference" / "SiO.out.121mpi"))
    kuu = sorted(spectrum(REF / "tests" / "reference" / "KuuMuu_eig.txt"))
    spectra = {"SiO": {"n": len(sio), "lowest": sio[:40], "highest": sio[-40:]},
               "KuuMuu": {"n": len(kuu), "lowest": kuu[:40], "highest": kuu[-40:]}}
    (HERE / "spectra.json").write_text(json.dumps(spectra, indent=1))
    subprocess.run(["make", "-C", str(ROOT / "oracle")], check=True, capture_output=True)
    exe = ROOT / "oracle" / "_bin" / "rng_golden"
    rng = {}
    for seed in (1, 2, 7, 12345, 4294967295):
        out = subprocess.run([str(exe), str(seed), "64"], check=True, capture_output=True, text=True)
        rng[str(seed)] = [float(x) for x in out.stdout.split()]
    (HERE / "mt19937.json").write_text(json.dumps(rng, indent=1))
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
