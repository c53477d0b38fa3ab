"""The device FP64 symmetric eigensolver (fe_syevd_f64, and fe_syevd_batched_f64
past its 96 x 96 Jacobi kernel) against numpy.linalg.eigh: eigenvalues within
1e-12 ||A||, residuals ||A Z - Z diag(W)|| within 1e-12 ||A||, Z^T Z = I within
1e-12, on random matrices, clustered and exactly repeated spectra, the identity, a
1D Laplacian and a Rayleigh-Ritz-like projection, for k from 1 to 1000."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def cases():
    rng = np.random.default_rng(0)
    out = []
    for k in (1, 2, 3, 20, 64, 320, 512, 1000):
        M = rng.standard_normal((k, k))
        out.append((f"random{k}", M + M.T))
    Q, _ = np.linalg.qr(rng.standard_normal((320, 320)))
    lam = np.sort(np.concatenate([np.linspace(-4, 1, 280), 1.0 + 1e-9 * np.arange(20), [0.5] * 20]))
    out.append(("projection320", (Q * lam) @ Q.T))
    Q, _ = np.linalg.qr(rng.standard_normal((60, 60)))
    out.append(("clusters60", (Q * np.repeat([1.0, 2.0, 2.0 + 1e-13, 3.0], 15)) @ Q.T))
    out.append(("identity40", np.eye(40)))
    out.append(("repeated_diag40", np.diag(np.repeat([0.5, -1.0], 20))))
    L = 2 * np.eye(200) - np.eye(200, k=1) - np.eye(200, k=-1)
    out.append(("laplacian200", L))
    return out


def check(A, w, Z):
    nrm = np.abs(A).sum(axis=1).max()
    ref = np.linalg.eigvalsh(A)
    k = A.shape[0]
    assert np.abs(w - ref).max() <= 1e-12 * nrm
    assert np.abs(A @ Z - Z * w[None, :]).max() <= 1e-12 * nrm
    assert np.abs(Z.T @ Z - np.eye(k)).max() <= 1e-12


@pytest.mark.parametrize("name,A", cases(), ids=[c[0] for c in cases()])
def test_syevd_matches_numpy(name, A):
    import fasteig_b200 as fe
    k = A.shape[0]
    lda = k + 3  # a leading dimension larger than k
    dA = torch.zeros((k, lda), dtype=torch.float64, device="cuda")  # column-major k x k, ld lda
    dA[:, :k] = torch.from_numpy(A.T.copy()).cuda()
    W = torch.zeros(k, dtype=torch.float64, device="cuda")
    info = torch.ones(1, dtype=torch.int32, device="cuda")
    need = fe.lib.fe_syevd_f64_workspace_bytes(k)
    ws = torch.empty(need, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = fe.lib.fe_syevd_f64(dA.data_ptr(), lda, k, W.data_ptr(), info.data_ptr(), ws.data_ptr(),
                             need, stream)
    assert rc == 0, fe.lib.fe_last_error().decode()
    torch.cuda.synchronize()
    assert int(info.item()) == 0
    Z = dA[:, :k].cpu().numpy().T  # column-major back to (row, col)
    check(A, W.cpu().numpy(), Z)


def test_syevd_nonfinite_input_sets_info():
    import fasteig_b200 as fe
    k = 8
    A = np.eye(k)
    A[3, 3] = np.nan
    dA = torch.from_numpy(A.copy()).cuda()
    W = torch.zeros(k, dtype=torch.float64, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    need = fe.lib.fe_syevd_f64_workspace_bytes(k)
    ws = torch.empty(need, dtype=torch.uint8, device="cuda")
    assert fe.lib.fe_syevd_f64(dA.data_ptr(), k, k, W.data_ptr(), info.data_ptr(), ws.data_ptr(),
                               need, None) == 0
    torch.cuda.synchronize()
    assert int(info.item()) == 1


def test_batched_syevd_past_jacobi_limit():
    import fasteig_b200 as fe
    rng = np.random.default_rng(5)
    sizes = [130, 20, 257]
    lda = max(sizes)
    mats = np.zeros((len(sizes), lda, lda))
    As = []
    for p, m in enumerate(sizes):
        M = rng.standard_normal((m, m))
        A = M + M.T
        As.append(A)
        mats[p, :m, :m] = A.T  # column-major block of matrix p
    dA = torch.from_numpy(mats).cuda()
    W = torch.zeros((len(sizes), lda), dtype=torch.float64, device="cuda")
    Z = torch.zeros_like(dA)
    m_arr = np.array(sizes, dtype=np.int32)
    rc = fe.lib.fe_syevd_batched_f64(len(sizes), m_arr.ctypes.data, dA.data_ptr(), lda,
                                     W.data_ptr(), Z.data_ptr(), None)
    assert rc == 0, fe.lib.fe_last_error().decode()
    Wh, Zh = W.cpu().numpy(), Z.cpu().numpy()
    for p, (m, A) in enumerate(zip(sizes, As)):
        check(A, Wh[p, :m], Zh[p, :m, :m].T)
    assert np.array_equal(dA.cpu().numpy(), mats)  # input untouched


@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("k", [32, 96, 160])
def test_syevd_tridiagonalization_kernels(mode, k):
    """Both tridiagonalization kernels (one CTA, 8-CTA cluster) give the spectrum of
    numpy.linalg.eigh to 1e-12 * ||A|| and orthonormal vectors."""
    import fasteig_b200 as fe
    rng = np.random.default_rng(k + mode)
    M = rng.standard_normal((k, k))
    A = M + M.T
    dA = torch.from_numpy(A.copy()).cuda()
    W = torch.zeros(k, dtype=torch.float64, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    need = fe.lib.fe_syevd_f64_workspace_bytes(k)
    ws = torch.empty(need, dtype=torch.uint8, device="cuda")
    assert fe.lib.fe_set_syevd_kernel(mode) == 0
    try:
        assert fe.lib.fe_syevd_f64(dA.data_ptr(), k, k, W.data_ptr(), info.data_ptr(),
                                   ws.data_ptr(), need, None) == 0
        torch.cuda.synchronize()
    finally:
        fe.lib.fe_set_syevd_kernel(0)
    assert int(info.item()) == 0
    scale = np.abs(A).sum(axis=1).max()
    assert np.abs(W.cpu().numpy() - np.linalg.eigvalsh(A)).max() <= 1e-12 * scale
    Z = dA.cpu().numpy().reshape(k, k).T  # column-major eigenvectors
    assert np.abs(Z.T @ Z - np.eye(k)).max() <= 1e-12 * k
