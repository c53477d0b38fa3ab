"""Failure detection without a GPU fault: every spin-wait in the tensor-core and
pipelined SpMM kernels is bounded and records a code in a device status word.

  * fe_selftest_wait_timeout makes one bounded wait run out (an mbarrier nothing
    arrives on, about a millisecond of SM clock): the code reaches the library's
    default word, fe_device_status reads and clears it, and later kernels run.
  * A solve records timeouts in a status word of its own: the fe_solve test hook
    inject_wait_timeout=<code> runs the same probe on that word; the solve fails with
    FE_ERR_CUDA naming the code, the default word stays clear, and the next solve
    is unaffected.
  * Two requests on the server at once, one with the hook: the code reaches that
    request only; the other returns the same eigenvalues as fe_solve alone.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _status(clear=True):
    import fasteig_b200 as fe
    v = C.c_int32()
    assert fe.lib.fe_device_status(C.byref(v), 1 if clear else 0) == 0
    return int(v.value)


def _opts(n, **kw):
    from fasteig_b200 import fasteig_options
    o = fasteig_options(n)
    base = dict(solver="Chebyshev", nev=6, which="SR", tol=1e-8, maxiter=400, seed=1, degree=8)
    base.update(kw)
    for k, v in base.items():
        assert o.set(k, v), k
    return o


@pytest.fixture(scope="module")
def wells():
    import fasteig_b200 as fe
    from fasteig_b200 import matrices as M
    H = M.laplacian_wells(10, wells=6, seed=1)
    return H, fe.CsrMatrix(H.n, H.rowptr, H.colind, H.values)


def test_selftest_wait_timeout_reaches_default_word():
    import fasteig_b200 as fe
    from fasteig_b200 import ops
    _status(clear=True)
    assert fe.lib.fe_selftest_wait_timeout(1_000_000, 91, None) == 0
    torch.cuda.synchronize()
    assert _status(clear=True) == 91
    assert _status(clear=False) == 0
    # the context is usable: a tensor-core Gram runs and records nothing
    X = torch.randn(4096, 64, device="cuda", dtype=torch.float32)
    G = ops.gram_tf32x3(X, X)
    torch.cuda.synchronize()
    ref = X.double().T @ X.double()
    assert float((G - ref).abs().max()) <= 1e-4 * float(ref.abs().max())
    assert _status(clear=False) == 0


def test_solve_timeout_reported_to_that_solve(wells):
    import fasteig_b200 as fe
    from fasteig_b200 import fasteig_problem
    H, dA = wells
    _status(clear=True)
    p = fasteig_problem(dA, solver="Chebyshev")
    with pytest.raises(fe.FastEigError, match="status code 77"):
        p.solve(_opts(H.n, inject_wait_timeout=77, precision="mixed"))
    assert _status(clear=False) == 0
    q = fasteig_problem(dA, solver="Chebyshev")
    q.solve(_opts(H.n))
    assert np.all(q.residual_norms() <= 1e-8)


def test_server_timeout_reaches_the_right_request(wells):
    import fasteig_b200 as fe
    from fasteig_b200 import fasteig_problem
    H, dA = wells
    alone = fasteig_problem(dA, solver="Chebyshev")
    alone.solve(_opts(H.n), want_vectors=False)
    with fe.Server(slots=2) as srv:
        bad = srv.submit(dA, _opts(H.n, inject_wait_timeout=78))
        good = srv.submit(dA, _opts(H.n))
        with pytest.raises(fe.FastEigError, match="status code 78"):
            srv.wait(bad)
        res = srv.wait(good)
    np.testing.assert_array_equal(res["eigenvalues"], alone.eigenvalues())
    assert _status(clear=False) == 0
