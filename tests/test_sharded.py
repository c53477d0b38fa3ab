"""Row-sharded Chebyshev solver (fasteig_b200/sharded.py).

CPU: the row partition and halo plan reproduce the global SpMM from local operators;
the driver runs on 2 and 3 ``gloo`` ranks (separate processes) with a NumPy backend of
the backend interface and matches the single-process oracle (oracle.chebyshev_solve,
the restatement of src/ChebyshevSolver.cpp:67-221) iteration by iteration: eigenvalues
within 1e-10 relative, the same cycle count within 1, residuals <= tol.
GPU: the same driver on one rank with the library's CUDA backend against the oracle.
"""
import json
import os
import socket

import numpy as np
import pytest


def _problem(side=10, wells=6, seed=1):
    from fasteig_b200 import matrices as M
    H = M.laplacian_wells(side, wells=wells, seed=seed)
    return H


class TorchCpuBackend:
    """NumPy/torch-CPU arithmetic with the interface of CudaShardBackend (test only)."""

    def __init__(self):
        import torch
        self.torch = torch

    def operator(self, plan):
        import scipy.sparse as sp
        return sp.csr_matrix((plan.values, plan.colind, plan.rowptr), shape=(plan.n_own, plan.n_ext))

    def block(self, rows, cols, ld=None):
        return self.torch.zeros((rows, cols), dtype=self.torch.float64)

    def from_host(self, a):
        return self.torch.from_numpy(np.array(a, dtype=np.float64, copy=True))

    def to_host(self, t):
        return t.detach().numpy().copy()

    def spmm(self, A, X_ext, Y, alpha):
        Y[:] = self.torch.from_numpy(alpha * (A @ X_ext.numpy()))

    def cheb_step(self, A, cur_ext, prev, out, alpha, gamma, beta):
        n = out.shape[0]
        r = alpha * (A @ cur_ext.numpy()) + gamma * cur_ext[:n].numpy()
        if beta != 0.0:
            r = r + beta * prev.numpy()
        out[:] = self.torch.from_numpy(r)

    def gram(self, X, Y):
        return X.T @ Y

    def rotate(self, X, C, Y, alpha=1.0, beta=0.0):
        C = self.from_host(C) if isinstance(C, np.ndarray) else C
        Y[:] = alpha * (X @ C) + (beta * Y if beta != 0.0 else 0.0)

    def colsq(self, X):
        return (X * X).sum(0)

    def residual_sq(self, AX, X, lam):
        R = AX - X * self.from_host(lam)[None, :]
        return (R * R).sum(0), (X * X).sum(0)

    def cholesky_upper(self, G):
        try:
            return np.linalg.cholesky(G).T
        except np.linalg.LinAlgError:
            return None

    def inv_upper(self, R):
        import scipy.linalg as sl
        return sl.solve_triangular(R, np.eye(R.shape[0]))

    def eigh(self, P):
        return np.linalg.eigh(P)


def test_partition_reproduces_global_spmm():
    from fasteig_b200.sharded import plan_partition
    H = _problem(9)
    A = __import__("scipy.sparse", fromlist=["csr_matrix"]).csr_matrix(
        (H.values, H.colind, H.rowptr), shape=(H.n, H.n))
    X = np.random.default_rng(0).standard_normal((H.n, 5))
    ref = A @ X
    for world in (1, 2, 3, 5):
        plans = plan_partition(H.n, H.rowptr, H.colind, H.values, world)
        assert plans[0].r0 == 0 and plans[-1].r1 == H.n
        out = np.zeros_like(ref)
        for p in plans:
            Xe = np.vstack([X[p.r0:p.r1], X[p.ghosts]])
            import scipy.sparse as sp
            Al = sp.csr_matrix((p.values, p.colind, p.rowptr), shape=(p.n_own, p.n_ext))
            out[p.r0:p.r1] = Al @ Xe
            # what every peer sends this rank is exactly this rank's ghost run from it
            for q, (first, count) in p.recvs.items():
                sent = plans[q].sends[p.rank] + plans[q].r0
                np.testing.assert_array_equal(sent, p.ghosts[first:first + count])
        np.testing.assert_array_equal(out, ref)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, kw, out_path):
    import torch.distributed as dist
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            init_method=f"tcp://127.0.0.1:{port}")
    try:
        from fasteig_b200.sharded import sharded_chebyshev_solve
        H = _problem()
        res = sharded_chebyshev_solve(H.n, H.rowptr, H.colind, H.values, rank=rank, world=world,
                                      backend=TorchCpuBackend(), **kw)
        vec = res.vectors.numpy()
        with open(f"{out_path}.{rank}", "w") as f:
            json.dump({"values": res.eigenvalues.tolist(), "rel": res.residual_norms.tolist(),
                       "iters": res.iterations, "r0": res.r0, "r1": res.r1,
                       "vec": vec.tolist()}, f)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,kw", [
    (2, dict(nev=8, degree=10, tol=1e-8, maxiter=300, seed=1, block=12)),
    (3, dict(nev=8, degree=10, tol=1e-8, maxiter=300, seed=2, block=12, bounds="ritz",
             amplification=1e6, locking="hard")),
])
def test_sharded_gloo_matches_oracle(tmp_path, world, kw):
    import torch.multiprocessing as mp
    from oracle import oracle as O
    out = str(tmp_path / "res")
    mp.start_processes(_worker, args=(world, _free_port(), kw, out), nprocs=world, join=True,
                       start_method="spawn")
    parts = [json.load(open(f"{out}.{r}")) for r in range(world)]
    H = _problem()
    A = O.Csr(H.n, H.n, H.rowptr, H.colind, H.values)
    ref = O.chebyshev_solve(A, **kw)
    for p in parts:  # every rank holds the same replicated small results
        np.testing.assert_allclose(p["values"], ref.eigenvalues, rtol=1e-10, atol=1e-12)
        assert abs(p["iters"] - ref.iterations) <= 1, (p["iters"], ref.iterations)
        assert max(p["rel"]) <= 1e-8
    X = np.vstack([np.array(p["vec"]) for p in parts])
    final = O.residual_norms(A, None, np.array(parts[0]["values"]), X)
    assert np.all(final <= 1.01e-8), final


@pytest.mark.gpu
def test_sharded_cuda_backend_one_rank_matches_oracle():
    import torch
    import torch.distributed as dist
    from fasteig_b200.sharded import CudaShardBackend, sharded_chebyshev_solve
    from oracle import oracle as O
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1,
                            init_method=f"tcp://127.0.0.1:{_free_port()}",
                            device_id=torch.device("cuda", 0))
    try:
        H = _problem(12, 8, 2)
        kw = dict(nev=10, degree=10, tol=1e-8, maxiter=300, seed=3, block=16, bounds="ritz",
                  amplification=1e6, locking="hard")
        res = sharded_chebyshev_solve(H.n, H.rowptr, H.colind, H.values,
                                      backend=CudaShardBackend(), **kw)
        A = O.Csr(H.n, H.n, H.rowptr, H.colind, H.values)
        ref = O.chebyshev_solve(A, **kw)
        np.testing.assert_allclose(res.eigenvalues, ref.eigenvalues, rtol=1e-10, atol=1e-12)
        assert abs(res.iterations - ref.iterations) <= 1
        final = O.residual_norms(A, None, res.eigenvalues, res.vectors.cpu().numpy())
        assert np.all(final <= 1.01e-8), final
    finally:
        dist.destroy_process_group()
