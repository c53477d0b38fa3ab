"""fe_lanczos_step (one device-resident step of KrylovSubspace::build_one,
src/core/KrylovSubspace.cpp:125-131) against the oracle's restatement of the same
step (oracle._Lanczos.step), for 20 steps on the SiO matrix and on a 3D well
problem: tridiagonal T, basis V and final residual norm to 1e-12 relative."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def run_device(A, f0, m):
    import fasteig_b200 as fe
    dA = fe.CsrMatrix(A.rows, A.rowptr, A.colind, A.values)
    n = A.rows
    ld = (m + 7) // 8 * 8
    V = torch.zeros((n, ld), dtype=torch.float64, device="cuda")
    f = torch.from_numpy(f0.copy()).cuda()
    fn = torch.tensor([np.linalg.norm(f0)], dtype=torch.float64, device="cuda")
    T = torch.zeros((m, m), dtype=torch.float64, device="cuda")  # column-major m x m
    need = fe.lib.fe_lanczos_workspace_bytes(n, m)
    ws = torch.empty(need, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for j in range(m):
        rc = fe.lib.fe_lanczos_step(dA.handle, V.data_ptr(), ld, m, j, f.data_ptr(), fn.data_ptr(),
                                    T.data_ptr(), m, ws.data_ptr(), need, stream)
        assert rc == 0, fe.lib.fe_last_error().decode()
    torch.cuda.synchronize()
    return V[:, :m].cpu().numpy(), T.cpu().numpy().T, float(fn.item())


@pytest.mark.parametrize("case", ["sio", "wells"])
def test_lanczos_step_matches_oracle(case, sio):
    from fasteig_b200 import matrices as M
    from oracle import oracle as O
    if case == "sio":
        A = sio
    else:
        H = M.laplacian_wells(14, wells=8, seed=5)
        A = O.Csr(H.n, H.n, H.rowptr, H.colind, H.values)
    m = 20
    f0 = O.random_vector(A.rows, 3)
    Hs = A.scipy()
    ref = O._Lanczos(lambda v: Hs @ v, f0, m, 3)
    for it in range(m):
        ref.step(it)
    V, T, fnorm = run_device(A, f0, m)
    scale = np.abs(ref.T).max()
    assert np.abs(T - ref.T).max() <= 1e-12 * scale
    assert np.abs(V - ref.V).max() <= 1e-11
    assert abs(fnorm - ref.beta_next) <= 1e-11 * scale
    # the recurrence A V = V T + f e_m^T holds on the device result
    AV = Hs @ V
    assert np.abs(AV[:, :m - 1] - V @ T[:, :m - 1]).max() <= 1e-11 * scale
