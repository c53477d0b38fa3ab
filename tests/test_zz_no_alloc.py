"""The FP64 Gram entry point that allocates nothing (fe_gram_f64_noalloc).

It exists for callers that cannot allocate device memory when they call this
library (their device memory is owned by their own pool, or the call sits on a
path where cudaMalloc is not allowed), so it keeps its split-K partial sums in a
fixed array inside the library instead of a caller workspace. This file is named
to be collected last; it must pass alone in a fresh process and after the rest.
It checks the entry point through the C ABI against fe_gram_f64 (the allocating
variant) on two calls in a row, with the tolerance the Gram tests use:
|G - G_ref| <= 1e-13 |X|^T |Y| componentwise.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _gram_allocating(X, Y):
    import fasteig_b200 as fe
    n, k = X.shape
    m = Y.shape[1]
    Gt = torch.empty((m, k), dtype=torch.float64, device="cuda")
    need = fe.lib.fe_gram_workspace_bytes(n, k, m)
    ws = torch.empty(max(need, 8), dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    assert fe.lib.fe_gram_f64(X.data_ptr(), X.stride(0), Y.data_ptr(), Y.stride(0), n, k, m,
                              Gt.data_ptr(), k, ws.data_ptr(), need, stream) == 0
    return Gt.T


def _gram_noalloc(X, Y):
    import fasteig_b200 as fe
    n, k = X.shape
    m = Y.shape[1]
    Gt = torch.empty((m, k), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = fe.lib.fe_gram_f64_noalloc(X.data_ptr(), X.stride(0), Y.data_ptr(), Y.stride(0), n, k, m,
                                    Gt.data_ptr(), k, stream)
    assert rc == 0, fe.lib.fe_last_error().decode()
    return Gt.T


@pytest.mark.parametrize("n,k,m", [(200000, 320, 320), (70001, 17, 130)])
def test_noalloc_gram_matches_allocating_gram_twice(n, k, m):
    g = torch.Generator().manual_seed(n + k)
    for call in range(2):  # the shared scratch keeps the previous call's contents
        X = torch.randn(n, k, generator=g, dtype=torch.float64).cuda()
        Y = torch.randn(n, m, generator=g, dtype=torch.float64).cuda()
        G0 = _gram_noalloc(X, Y).cpu().numpy()
        G1 = _gram_allocating(X, Y).cpu().numpy()
        torch.cuda.synchronize()
        scale = np.abs(X.cpu().numpy()).T @ np.abs(Y.cpu().numpy())
        assert np.all(np.abs(G0 - G1) <= 1e-13 * scale), call


def test_noalloc_gram_at_its_exact_capacity():
    """k * m equal to the scratch size: one row chunk fills the whole array, where the
    allocating Gram splits the same rows over several chunks."""
    import fasteig_b200 as fe
    assert fe.lib.fe_gram_f64_noalloc_max_entries() == 1024 * 1024
    g = torch.Generator().manual_seed(11)
    n = 60000
    for call in range(2):
        X = torch.randn(n, 1024, generator=g, dtype=torch.float64).cuda()
        Y = X if call == 0 else torch.randn(n, 1024, generator=g, dtype=torch.float64).cuda()
        G0 = _gram_noalloc(X, Y).cpu().numpy()
        G1 = _gram_allocating(X, Y).cpu().numpy()
        torch.cuda.synchronize()
        scale = np.abs(X.cpu().numpy()).T @ np.abs(Y.cpu().numpy())
        assert np.all(np.abs(G0 - G1) <= 1e-13 * scale), call


def test_noalloc_gram_rejects_sizes_beyond_its_scratch():
    import fasteig_b200 as fe
    cap = fe.lib.fe_gram_f64_noalloc_max_entries()
    assert cap == 1 << 20
    X = torch.zeros(64, 1025, dtype=torch.float64, device="cuda")
    out = torch.zeros(1025 * 1025, dtype=torch.float64, device="cuda")
    rc = fe.lib.fe_gram_f64_noalloc(X.data_ptr(), 1025, X.data_ptr(), 1025, 64, 1025, 1025,
                                    out.data_ptr(), 1025, None)
    assert rc == -1
    assert "exceeds the static Gram scratch" in fe.lib.fe_last_error().decode()
