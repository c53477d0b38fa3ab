"""Compiled consumers of the C ABI: a C99 program (tests/cpp/consumer.c) and the
fasteig_problem::solve branch of INTEGRATION.md built against stand-ins of the
reference types (tests/cpp/fasteig_adapter.cpp), both linked to
fasteig_b200/libfasteig_b200.so. On the CPU they must compile and link (every symbol
they use is exported); on the GPU each solves SiO (n = 33,401) for its 5 lowest
eigenvalues with Chebyshev, LOBPCG, Davidson and Krylov-Schur and checks them against
the reference's ScaLAPACK spectrum (tests/reference/SiO.out.121mpi) with the
harness rule |dl| <= 1e-10 + 1e-10 |l|."""
import re
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
CPP = ROOT / "tests" / "cpp"
LIBDIR = ROOT / "fasteig_b200"

pytestmark = pytest.mark.skipif(shutil.which("gcc") is None or shutil.which("g++") is None,
                                reason="gcc/g++ not available")


def _build(tmp_path, src, lang):
    exe = tmp_path / src.stem
    cc = ["gcc", "-std=c99"] if lang == "c" else ["g++", "-std=c++17"]
    cmd = cc + ["-O1", "-Wall", "-Werror", "-I", str(ROOT / "include"), str(src), "-o", str(exe),
                "-L", str(LIBDIR), "-lfasteig_b200", f"-Wl,-rpath,{LIBDIR}",
                "-Wl,--allow-shlib-undefined", "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return exe


@pytest.fixture(scope="module")
def binaries(tmp_path_factory):
    d = tmp_path_factory.mktemp("cpp")
    return {"consumer": _build(d, CPP / "consumer.c", "c"),
            "adapter": _build(d, CPP / "fasteig_adapter.cpp", "c++")}


def test_consumers_compile_and_link(binaries):
    for exe in binaries.values():
        assert exe.exists()


def test_integration_doc_shows_the_compiled_branch():
    """The branch printed in INTEGRATION.md is the one compiled here."""
    src = (CPP / "fasteig_adapter.cpp").read_text()
    branch = src.split("// BEGIN fe_solve branch\n")[1].split("// END fe_solve branch")[0]
    doc = (ROOT / "INTEGRATION.md").read_text()
    block = re.search(r"```cpp\n(.*?)```", doc, re.S).group(1)
    code = lambda t: [ln.strip() for ln in t.splitlines()
                      if ln.strip() and not ln.strip().startswith(("#include", "//"))]
    assert code(block) == code(branch)


def _input_file(tmp_path, sio, spectra):
    exp = np.array(spectra["SiO"]["lowest"][:5])
    path = tmp_path / "sio.bin"
    with open(path, "wb") as f:
        np.array([sio.rows, sio.values.size, exp.size], dtype=np.int64).tofile(f)
        sio.rowptr.astype(np.int32).tofile(f)
        sio.colind.astype(np.int32).tofile(f)
        sio.values.astype(np.float64).tofile(f)
        exp.astype(np.float64).tofile(f)
    return path


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["consumer", "adapter"])
def test_compiled_consumer_solves_sio(binaries, tmp_path, sio, spectra, which):
    inp = _input_file(tmp_path, sio, spectra)
    solvers = ["chebyshev", "lobpcg", "davidson", "krylovschur"] if which == "consumer" else \
        ["Chebyshev", "LOBPCG", "Davidson", "KrylovSchur"]
    r = subprocess.run([str(binaries[which]), str(inp), *solvers], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
