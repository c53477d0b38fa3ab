"""Host tridiagonal eigensolver of the Lanczos snapshot (fasteig_b200/csrc/tridiag.hpp:
bisection on Sturm counts, inverse iteration with cluster reorthogonalization),
compiled with g++ through tests/cpp/tridiag_check.cpp and checked against
scipy.linalg.eigh_tridiagonal: eigenvalues to 1e-13 ||T||, residuals of the vectors to
1e-12 ||T||, orthonormality to 1e-10, on random, graded, split (zero coupling),
Wilkinson (close pairs) and Lanczos (the oracle's chain on SiO) tridiagonals; and the
snapshot's shortcut (bisection only for the eigenvalues a selection of nev pairs by
sr/lr/sm/lm/be can draw from) selects what the full spectrum selects."""
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest
import scipy.linalg as sla

ROOT = Path(__file__).resolve().parents[1]
pytestmark = pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    out = tmp_path_factory.mktemp("tri") / "tridiag_check"
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror",
                        str(ROOT / "tests" / "cpp" / "tridiag_check.cpp"), "-o", str(out)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return out


def run(exe, d, e):
    m = len(d)
    text = f"{m}\n" + " ".join(repr(float(x)) for x in d) + "\n" + \
        " ".join(repr(float(x)) for x in e) + "\n"
    r = subprocess.run([str(exe)], input=text, capture_output=True, text=True, check=True)
    lines = r.stdout.split("\n")
    w = np.array([float(x) for x in lines[:m]])
    V = np.array([[float(x) for x in ln.split()] for ln in lines[m:2 * m]]).T
    sel = [ln.split() for ln in lines[2 * m:] if ln.startswith("select")]
    assert sel and all(s[3] == "1" for s in sel), [s for s in sel if s[3] != "1"]
    return w, V


def check(exe, d, e):
    d, e = np.asarray(d, float), np.asarray(e, float)
    w, V = run(exe, d, e)
    ref = sla.eigh_tridiagonal(d, e, eigvals_only=True)
    T = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
    tn = np.abs(T).sum(axis=1).max()
    assert np.abs(w - ref).max() <= 1e-13 * tn
    assert np.abs(T @ V - V * w).max() <= 1e-12 * tn
    assert np.abs(V.T @ V - np.eye(len(d))).max() <= 1e-10


def test_random_and_graded(exe):
    rng = np.random.default_rng(0)
    for m in (1, 2, 7, 60):
        check(exe, rng.standard_normal(m), rng.standard_normal(m - 1))
    m = 40
    check(exe, 10.0 ** np.linspace(-6, 6, m), 10.0 ** np.linspace(-6, 5, m - 1))


def test_split_and_wilkinson(exe):
    d = np.array([1.0, 2.0, 3.0, 1.0, 2.0, 3.0])
    e = np.array([0.5, 0.5, 0.0, 0.5, 0.5])  # two equal decoupled blocks: double eigenvalues
    check(exe, d, e)
    k = 10  # Wilkinson W21+: pairs agreeing to many digits
    check(exe, np.abs(np.arange(-k, k + 1, dtype=float)), np.ones(2 * k))


def test_lanczos_chain_of_sio(exe, sio):
    from oracle import oracle as O
    lz = O._Lanczos(lambda v: sio.scipy() @ v, O.random_vector(sio.rows, 1), 120, 1)
    for it in range(120):
        lz.step(it)
    T = lz.T
    check(exe, np.diag(T), np.diag(T, -1))
