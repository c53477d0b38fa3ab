"""FP64 Gram and rotation on both kernel families (FP64 tensor-core DMMA, the
default, and SIMT FP64 FMA) through the C ABI, against the FP64 oracle product:

  Gram:      |G - X^T Y| <= 1e-13 |X|^T |Y|      (symmetric X^T X exactly symmetric)
  Rotation:  |Y - (a X C + b Y0)| <= 1e-13 (|a| |X||C| + |b| |Y0|)

Shapes cover the ragged edges of the 64-wide tiles, row chunks that end inside a
16-row stage, column views that start off a 16-byte boundary (8-byte copies)
and leading dimensions that are odd.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(params=[0, 1], ids=["dmma", "simt"])
def f64_kernel(request):
    import fasteig_b200 as fe
    assert fe.lib.fe_set_f64_gemm_kernel(request.param) == 0
    yield request.param
    assert fe.lib.fe_set_f64_gemm_kernel(0) == 0


def view(n, cols, seed, ld=None, offset=0):
    """n x cols FP64 view into an n x ld buffer starting at column `offset`."""
    ld = ld or cols + offset
    g = torch.Generator().manual_seed(seed)
    base = torch.randn(n, ld, generator=g, dtype=torch.float64).cuda()
    return base[:, offset:offset + cols]


SHAPES = [(1, 1, 1, 0), (5, 3, 2, 0), (37, 9, 7, 1), (1000, 17, 33, 0), (4097, 64, 64, 0),
          (20011, 65, 130, 3), (70001, 130, 70, 0), (9000, 320, 320, 0), (3001, 320, 320, 1)]


@pytest.mark.parametrize("n,k,m,off", SHAPES)
def test_gram_f64_kernels(f64_kernel, n, k, m, off):
    from fasteig_b200 import ops
    X = view(n, k, 11, offset=off)
    Y = view(n, m, 12, ld=m + 5)
    G = ops.gram(X, Y).cpu().numpy()
    X64, Y64 = X.cpu().numpy(), Y.cpu().numpy()
    ref = X64.T @ Y64
    scale = np.abs(X64).T @ np.abs(Y64)
    assert np.all(np.abs(G - ref) <= 1e-13 * scale + 1e-300)


@pytest.mark.parametrize("n,k,off", [(7, 5, 0), (1000, 64, 0), (5003, 130, 1), (20000, 320, 0),
                                     (4099, 200, 3)])
def test_gram_f64_symmetric(f64_kernel, n, k, off):
    from fasteig_b200 import ops
    X = view(n, k, 13, offset=off)
    G = ops.gram(X, X).cpu().numpy()
    X64 = X.cpu().numpy()
    ref = X64.T @ X64
    scale = np.abs(X64).T @ np.abs(X64)
    assert np.all(np.abs(G - ref) <= 1e-13 * scale + 1e-300)
    assert np.array_equal(G, G.T)


def test_gram_f64_kernels_deterministic(f64_kernel):
    from fasteig_b200 import ops
    X = view(60000, 96, 14)
    G1 = ops.gram(X, X).clone()
    G2 = ops.gram(X, X)
    assert torch.equal(G1, G2)


@pytest.mark.parametrize("n,k,m,off", SHAPES)
@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (-0.5, 2.0)])
def test_rotate_f64_kernels(f64_kernel, n, k, m, off, alpha, beta):
    from fasteig_b200 import ops
    X = view(n, k, 21, offset=off)
    Y = view(n, m, 22, ld=m + 3)
    Cm = torch.randn(k, m, dtype=torch.float64, generator=torch.Generator().manual_seed(5)).cuda()
    X64, Y64, C64 = X.cpu().numpy(), Y.cpu().numpy(), Cm.cpu().numpy()
    ref = alpha * X64 @ C64 + beta * Y64
    ops.rotate(X, Cm, Y, alpha, beta)
    scale = abs(alpha) * np.abs(X64) @ np.abs(C64) + abs(beta) * np.abs(Y64)
    assert np.all(np.abs(Y.cpu().numpy() - ref) <= 1e-13 * scale + 1e-300)


def test_gram_noalloc_uses_both_kernels(f64_kernel):
    import fasteig_b200 as fe
    X = view(30000, 80, 31)
    Gt = torch.empty((80, 80), dtype=torch.float64, device="cuda")
    rc = fe.lib.fe_gram_f64_noalloc(X.data_ptr(), X.stride(0), X.data_ptr(), X.stride(0),
                                    30000, 80, 80, Gt.data_ptr(), 80, None)
    assert rc == 0
    torch.cuda.synchronize()
    X64 = X.cpu().numpy()
    ref = X64.T @ X64
    assert np.all(np.abs(Gt.T.cpu().numpy() - ref) <= 1e-13 * (np.abs(X64).T @ np.abs(X64)))
