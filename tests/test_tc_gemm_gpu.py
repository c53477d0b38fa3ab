"""tcgen05 split-TF32 Gram and rotation against FP64 references.

Tolerance (componentwise): |G - G_ref| <= 4e-6 |X|^T|Y| for the Gram (3xTF32
products carry ~2^-22 relative error, FP32 accumulation per 32-row block, FP64
across chunks), |Y - Y_ref| <= (k + 4) 2^-22 (|X||C| + |beta||Y|) for the rotation.
Each test also checks the device status word of the bounded waits."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def blk(n, b, seed, ld=None):
    g = torch.Generator().manual_seed(seed)
    ld = ld or b
    t = torch.randn(n, ld, generator=g, dtype=torch.float64).float().cuda()
    return t[:, :b] if ld != b else t


@pytest.mark.parametrize("n,k,m", [(128, 8, 8), (1000, 17, 33), (4096, 128, 160), (5000, 160, 128),
                                   (33333, 64, 320), (70001, 320, 320), (2048, 300, 5)])
def test_gram_tf32x3(n, k, m):
    from fasteig_b200 import ops
    assert ops.device_status(clear=True) == 0
    X = blk(n, k, 1, ld=((k + 3) // 4) * 4)
    Y = blk(n, m, 2, ld=((m + 3) // 4) * 4)
    G = ops.gram_tf32x3(X, Y)
    torch.cuda.synchronize()
    assert ops.device_status() == 0
    X64, Y64 = X.double().cpu().numpy(), Y.double().cpu().numpy()
    ref = X64.T @ Y64
    scale = np.abs(X64).T @ np.abs(Y64)
    err = np.abs(G.cpu().numpy() - ref)
    assert np.all(err <= 4e-6 * scale + 1e-30), (err / scale).max()


def test_gram_tf32x3_column_offset_views():
    from fasteig_b200 import ops
    base = blk(9000, 64, 3)
    X = base[:, 0:13]       # aligned start
    Y = base[:, 13:50]      # start not 16-byte aligned: shifted tensor map
    G = ops.gram_tf32x3(X, Y)
    torch.cuda.synchronize()
    X64, Y64 = X.double().cpu().numpy(), Y.double().cpu().numpy()
    np.testing.assert_allclose(G.cpu().numpy(), X64.T @ Y64, rtol=0,
                               atol=4e-6 * (np.abs(X64).T @ np.abs(Y64)).max())


def test_gram_tf32x3_deterministic():
    from fasteig_b200 import ops
    X = blk(100000, 96, 4)
    assert torch.equal(ops.gram_tf32x3(X, X).clone(), ops.gram_tf32x3(X, X))


@pytest.mark.parametrize("n,k,m", [(128, 8, 8), (1000, 17, 33), (4100, 320, 320), (777, 64, 160),
                                   (20000, 256, 320), (3000, 5, 300)])
@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (-1.0, 1.0)])
def test_rotate_tf32x3(n, k, m, alpha, beta):
    from fasteig_b200 import ops
    assert ops.device_status(clear=True) == 0
    X = blk(n, k, 5, ld=((k + 3) // 4) * 4)
    Y = blk(n, m, 6)
    Cm = torch.randn(k, m, dtype=torch.float64, generator=torch.Generator().manual_seed(7)).cuda()
    X64, Y64, C64 = X.double().cpu().numpy(), Y.double().cpu().numpy(), Cm.cpu().numpy()
    ref = alpha * X64 @ C64 + (beta * Y64 if beta else 0.0)
    ops.rotate_tf32x3(X, Cm, Y, alpha, beta)
    torch.cuda.synchronize()
    assert ops.device_status() == 0
    scale = np.abs(X64) @ np.abs(C64) + (abs(beta) * np.abs(Y64) if beta else 0.0)
    err = np.abs(Y.double().cpu().numpy() - ref)
    assert np.all(err <= (k + 4) * 2.0 ** -22 * scale + 1e-30), (err / scale).max()


def test_rotate_tf32x3_output_column_view():
    from fasteig_b200 import ops
    V = blk(5000, 40, 8)
    Cm = torch.randn(13, 27, dtype=torch.float64).cuda()
    ref = V[:, :13].double() @ Cm * -1.0 + V[:, 13:40].double()
    ops.rotate_tf32x3(V[:, :13], Cm, V[:, 13:40], -1.0, 1.0)  # X - V*H into the next columns
    torch.cuda.synchronize()
    np.testing.assert_allclose(V[:, 13:40].double().cpu().numpy(), ref.cpu().numpy(),
                               rtol=0, atol=2e-5 * np.abs(ref.cpu().numpy()).max())


@pytest.mark.parametrize("locked,sub", [(250, 320), (253, 320), (130, 320), (97, 300)])
def test_rotate_tf32x3_deflation_update_in_place(locked, sub):
    """The Chebyshev deflation update V[:, locked:] -= V[:, :locked] G inside one
    320-wide slab: output column view at any offset (not 16-byte aligned)."""
    from fasteig_b200 import ops
    assert ops.device_status(clear=True) == 0
    V = blk(20011, sub, 9, ld=320)
    G = torch.randn(locked, sub - locked, dtype=torch.float64,
                    generator=torch.Generator().manual_seed(3)).cuda() * 0.1
    V64 = V.double().cpu().numpy()
    ref = V64[:, locked:] - V64[:, :locked] @ G.cpu().numpy()
    ops.rotate_tf32x3(V[:, :locked], G, V[:, locked:], -1.0, 1.0)
    torch.cuda.synchronize()
    assert ops.device_status() == 0
    scale = np.abs(V64[:, :locked]) @ np.abs(G.cpu().numpy()) + np.abs(V64[:, locked:])
    err = np.abs(V[:, locked:].double().cpu().numpy() - ref)
    assert np.all(err <= (locked + 4) * 2.0 ** -22 * scale + 1e-30), (err / scale).max()
    # untouched locked columns
    assert np.array_equal(V[:, :locked].double().cpu().numpy(), V64[:, :locked])


@pytest.fixture(params=[0, 1, 2], ids=["persistent_tmem_a", "per_tile", "persistent_smem_split"])
def rotate_kernel(request):
    import fasteig_b200 as fe
    assert fe.lib.fe_set_tc_rotate_kernel(request.param) == 0
    yield request.param
    assert fe.lib.fe_set_tc_rotate_kernel(0) == 0


@pytest.mark.parametrize("n,k,m", [(128, 8, 8), (20000, 256, 320), (70001, 320, 320),
                                   (33333, 320, 200), (131072, 64, 160)])
@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (-1.0, 1.0)])
def test_rotate_tf32x3_both_kernels(rotate_kernel, n, k, m, alpha, beta):
    """The persistent rotations (several tiles per CTA, alternating TMEM accumulators;
    X split in registers and read by the MMA from TMEM, or split in shared memory) and
    the one-CTA-per-tile rotation give the same product within the 3xTF32 bound, and are
    bit-identical to each other (same MMAs, same order)."""
    import fasteig_b200 as fe
    from fasteig_b200 import ops
    assert ops.device_status(clear=True) == 0
    X = blk(n, k, 15, ld=((k + 3) // 4) * 4)
    Y = blk(n, m, 16)
    Y0 = Y.clone()
    Cm = torch.randn(k, m, dtype=torch.float64, generator=torch.Generator().manual_seed(2)).cuda()
    X64, Y64, C64 = X.double().cpu().numpy(), Y.double().cpu().numpy(), Cm.cpu().numpy()
    ref = alpha * X64 @ C64 + (beta * Y64 if beta else 0.0)
    ops.rotate_tf32x3(X, Cm, Y, alpha, beta)
    torch.cuda.synchronize()
    assert ops.device_status() == 0
    scale = np.abs(X64) @ np.abs(C64) + (abs(beta) * np.abs(Y64) if beta else 0.0)
    err = np.abs(Y.double().cpu().numpy() - ref)
    assert np.all(err <= (k + 4) * 2.0 ** -22 * scale + 1e-30), (err / scale).max()
    for other in {0, 1, 2} - {rotate_kernel}:
        assert fe.lib.fe_set_tc_rotate_kernel(other) == 0
        Y2 = Y0.clone()
        ops.rotate_tf32x3(X, Cm, Y2, alpha, beta)
        torch.cuda.synchronize()
        assert torch.equal(Y, Y2), other


@pytest.mark.parametrize("n,k,off", [(5000, 320, 0), (33333, 300, 1), (4096, 400, 3), (777, 130, 2)])
def test_gram_tf32x3_symmetric_mirrored_tiles(n, k, off):
    """X^T X skips the tiles wholly below the diagonal and mirrors them in the FP64
    reduction: the mirrored entries equal their transposes and every entry keeps the
    split-TF32 bound, also for a column view that does not start on a 16-byte boundary."""
    from fasteig_b200 import ops
    assert ops.device_status(clear=True) == 0
    V = blk(n, k + off, 21, ld=((k + off + 3) // 4) * 4)
    X = V[:, off:off + k]
    G = ops.gram_tf32x3(X, X).cpu().numpy()
    torch.cuda.synchronize()
    assert ops.device_status() == 0
    X64 = X.double().cpu().numpy()
    ref = X64.T @ X64
    scale = np.abs(X64).T @ np.abs(X64)
    assert np.all(np.abs(G - ref) <= 4e-6 * scale + 1e-30), (np.abs(G - ref) / scale).max()
    i, j = np.indices(G.shape)
    mirrored = ((i + off) // 128) * 128 >= ((j + off) // 160) * 160 + 160
    assert np.array_equal(G[mirrored], G.T[mirrored])


@pytest.mark.parametrize("n,k", [(1_000_000, 128), (600_000, 320)])
def test_gram_tf32x3_long_row_chunks_keep_bound(n, k):
    """Row chunks of thousands of rows per CTA: the tensor cores' FP32 accumulator is
    restarted every 256 rows and summed in FP32 registers, so the componentwise bound
    holds at any n (before, the diagonal's error grew with the chunk length: 3.3e-4
    relative at n = 2,097,152)."""
    from fasteig_b200 import ops
    assert ops.device_status(clear=True) == 0
    g = torch.Generator(device="cuda").manual_seed(n + k)
    X = torch.randn(n, k, device="cuda", dtype=torch.float32, generator=g)
    G = ops.gram_tf32x3(X, X)
    torch.cuda.synchronize()
    assert ops.device_status() == 0
    X64 = X.double()
    ref = X64.T @ X64
    scale = X64.abs().T @ X64.abs()
    rel = ((G.double() - ref).abs() / scale).max().item()
    assert rel <= 4e-6, rel
