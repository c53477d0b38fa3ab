"""C ABI library checks that need no GPU: it loads, exports every entry point
include/fasteig_b200.h declares, and rejects invalid arguments with status
codes (validation happens before any device work)."""
import ctypes as C
import re

import numpy as np
import pytest

from conftest import ROOT


def declared_symbols():
    hdr = (ROOT / "include" / "fasteig_b200.h").read_text()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(fe_[a-z0-9_]+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol():
    import fasteig_b200 as fe
    names = declared_symbols()
    assert len(names) >= 25
    for name in names:
        assert hasattr(fe.lib, name), name
    # and the ctypes binding table covers them
    from fasteig_b200._lib import EXPORTED
    assert set(names) <= set(EXPORTED)


def test_version_and_error_reporting():
    import fasteig_b200 as fe
    assert "sm_100a" in fe.version()
    assert fe.lib.fe_csr_destroy(None) == 0


def _csr_create(n, rowptr, colind, vals, cols=None):
    import fasteig_b200 as fe
    h = C.c_void_p()
    rp = np.ascontiguousarray(rowptr, dtype=np.int32)
    ci = np.ascontiguousarray(colind, dtype=np.int32)
    v = np.ascontiguousarray(vals, dtype=np.float64)
    st = fe.lib.fe_csr_create(n, n if cols is None else cols, v.size, rp.ctypes.data,
                              ci.ctypes.data if ci.size else None,
                              v.ctypes.data if v.size else None, C.byref(h))
    return st, fe.lib.fe_last_error().decode()


@pytest.mark.parametrize("rowptr,colind,msg", [
    ([1, 1, 2], [0, 1], "rowptr must start at zero"),
    ([0, 1, 3], [0, 1], "rowptr end must equal nnz"),
    ([0, 2, 1], [0], "nondecreasing"),
    ([0, 2, 1, 2], [0, 1], "nondecreasing"),
    ([0, 1, 2], [0, 5], "column index out of range"),
    ([0, 1, 2], [-1, 0], "column index out of range"),
])
def test_csr_validation_matches_reference_messages(rowptr, colind, msg):
    n = len(rowptr) - 1
    st, err = _csr_create(n, rowptr, colind, np.ones(len(colind)))
    assert st == -1
    assert msg in err


def test_solve_rejects_null_handle_and_bad_options():
    import fasteig_b200 as fe
    vals = np.zeros(4)
    res = np.zeros(4)
    st = fe.lib.fe_solve(None, None, b"nev=4", vals.ctypes.data, res.ctypes.data, None, None)
    assert st == -1 and "null CSR handle" in fe.lib.fe_last_error().decode()


def test_workspace_queries_are_host_only():
    import fasteig_b200 as fe
    assert fe.lib.fe_gram_workspace_bytes(2097152, 320, 320) > 0
    assert fe.lib.fe_gram_workspace_bytes(0, 3, 3) == 0
    assert fe.lib.fe_residual_workspace_bytes(1000, 17) >= 2 * 17 * 8


def test_extension_options_reach_the_option_text():
    """Extension keys (locking, precision, mixed_switch) are accepted and passed to
    fe_solve's option text; unknown keys are refused like the reference's set()."""
    import fasteig_b200 as fe
    o = fe.fasteig_options(100)
    for k, v in (("solver", "Chebyshev"), ("locking", "hard"), ("precision", "mixed"),
                 ("mixed_switch", 1e-6)):
        assert o.set(k, v), k
    text = o.to_text()
    for frag in ("locking=hard", "precision=mixed", "mixed_switch=1e-06"):
        assert frag in text, (frag, text)
    assert not o.set("no_such_option", 1)
