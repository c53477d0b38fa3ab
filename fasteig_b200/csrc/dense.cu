// Small FP64 dense kernels that keep the k-by-k steps of Cholesky QR on the
// device: upper Cholesky factorization with a device-side rank-loss flag,
// triangular inverse, symmetrization. Also the CSR object, error reporting and
// library identity of the C ABI.
//
// Replaces cusolverDnDpotrf + the info device-to-host copy + stream sync and
// the cublasDtrsm of cuda_cholesky_qr_in_place (src/core/Orthogonalization.cpp:
// 185-246). The reference's rank-loss return (-1 when potrf reports info > 0,
// :224) becomes a device int that the host reads together with the other
// per-iteration scalars.

#include "fe_common.cuh"

#include <atomic>
#include <map>
#include <cmath>
#include <mutex>
#include <string>
#include <vector>

namespace fe {

namespace {
thread_local std::string g_last_error;
}

void set_last_error(const std::string& msg) { g_last_error = msg; }

namespace {
std::atomic<int64_t> g_launches{0};
}
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

namespace {
thread_local int* tl_status_word = nullptr;
}
int* current_status_word() { return tl_status_word; }
void set_status_word(int* word) { tl_status_word = word; }

int* thread_status_word() {
  constexpr int kDevices = 64;
  thread_local int* words[kDevices] = {};
  int dev = 0;
  FE_CHECK_CUDA(cudaGetDevice(&dev));
  FE_REQUIRE(dev >= 0 && dev < kDevices, "device index out of range");
  int*& w = words[dev];
  if (w) {
    // Still this device's memory? (not after cudaDeviceReset)
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, w) != cudaSuccess || a.type != cudaMemoryTypeDevice ||
        a.device != dev) {
      (void)cudaGetLastError();
      w = nullptr;
    }
  }
  if (!w) FE_CHECK_CUDA(cudaMalloc(&w, sizeof(int)));
  return w;
}

cudaStream_t& alloc_stream() {
  thread_local cudaStream_t s = nullptr;
  return s;
}

void retain_pool_memory(int device) {
  static std::mutex mu;
  static bool done[64] = {};
  if (device < 0 || device >= 64) return;
  std::lock_guard<std::mutex> lock(mu);
  if (done[device]) return;
  cudaMemPool_t pool;
  FE_CHECK_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
  uint64_t keep = UINT64_MAX;
  FE_CHECK_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
  done[device] = true;
}

// ---- cache of large solve buffers --------------------------------------------
// A solve allocates a handful of multi-GB blocks whose sizes repeat from one solve
// of a configuration to the next. They are kept after release and handed back to
// a request of the same (2 MiB-rounded) size on the same device: the release
// records an event on its stream and the next user's stream waits on it, so reuse
// is stream-ordered. A failed allocation first returns the cached blocks to the
// device and retries.
namespace {
struct CachedBlock {
  void* ptr;
  cudaEvent_t ready;
};
std::mutex g_cache_mutex;
std::map<std::pair<int, size_t>, std::vector<CachedBlock>> g_cache;

size_t round_block(size_t bytes) {
  const size_t g = size_t(2) << 20;
  return (bytes + g - 1) / g * g;
}

void trim_cache(int device) {
  std::vector<CachedBlock> drop;
  {
    std::lock_guard<std::mutex> lock(g_cache_mutex);
    for (auto it = g_cache.begin(); it != g_cache.end();) {
      if (it->first.first == device) {
        drop.insert(drop.end(), it->second.begin(), it->second.end());
        it = g_cache.erase(it);
      } else {
        ++it;
      }
    }
  }
  for (auto& b : drop) {
    cudaEventSynchronize(b.ready);
    cudaEventDestroy(b.ready);
    cudaFree(b.ptr);
  }
}

// The stream-ordered pool keeps what solves freed (release threshold: all of it);
// return the unused part to the device.
void trim_pool(int device) {
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
}
}  // namespace

void release_cached_memory(int device) {
  trim_cache(device);
  trim_pool(device);
}

void* big_alloc(size_t bytes, cudaStream_t s, size_t* granted) {
  int dev = 0;
  FE_CHECK_CUDA(cudaGetDevice(&dev));
  const size_t want = round_block(bytes);
  *granted = want;
  {
    std::lock_guard<std::mutex> lock(g_cache_mutex);
    auto it = g_cache.find({dev, want});
    if (it != g_cache.end() && !it->second.empty()) {
      CachedBlock b = it->second.back();
      it->second.pop_back();
      cudaError_t e = cudaStreamWaitEvent(s, b.ready, 0);
      cudaEventDestroy(b.ready);
      if (e != cudaSuccess) {
        cudaFree(b.ptr);
        FE_CHECK_CUDA(e);
      }
      return b.ptr;
    }
  }
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, want);
  if (e != cudaSuccess) {
    cudaGetLastError();
    release_cached_memory(dev);
    e = cudaMalloc(&p, want);
  }
  if (e != cudaSuccess) {
    throw Error(FE_ERR_ALLOC, std::string("cudaMalloc(") + std::to_string(want) +
                                  ") failed: " + cudaGetErrorString(e));
  }
  return p;
}

void big_free(void* p, size_t granted, cudaStream_t s) {
  int dev = 0;
  cudaEvent_t ev = nullptr;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventRecord(ev, s) != cudaSuccess) {
    if (ev) cudaEventDestroy(ev);
    cudaStreamSynchronize(s);
    cudaFree(p);
    return;
  }
  std::lock_guard<std::mutex> lock(g_cache_mutex);
  g_cache[{dev, granted}].push_back({p, ev});
}

int num_sms() {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 148;
  return sms > 0 ? sms : 148;
}

namespace {

// Right-looking unblocked Cholesky in one CTA. G is column-major (ldg); on
// return its upper triangle holds R (G = R^T R) and the strict lower part is 0.
__global__ void __launch_bounds__(1024)
potrf_upper_kernel(double* G, int k, int64_t ldg, int32_t* info) {
  __shared__ double inv_pivot;
  __shared__ int failed;
  if (threadIdx.x == 0) failed = 0;
  __syncthreads();
  for (int j = 0; j < k; ++j) {
    if (threadIdx.x == 0) {
      const double d = G[static_cast<int64_t>(j) * ldg + j];
      if (!(d > 0.0) || !isfinite(d)) {
        failed = j + 1;
      } else {
        const double r = sqrt(d);
        G[static_cast<int64_t>(j) * ldg + j] = r;
        inv_pivot = 1.0 / r;
      }
    }
    __syncthreads();
    if (failed) break;
    // Row j of R: R[j][c] = G[j][c] / r_jj for c > j.
    for (int c = j + 1 + threadIdx.x; c < k; c += blockDim.x) {
      G[static_cast<int64_t>(c) * ldg + j] *= inv_pivot;
    }
    __syncthreads();
    // Trailing update of the upper triangle: G[a][c] -= R[j][a] R[j][c], j < a <= c.
    const int t = k - j - 1;
    const int64_t count = static_cast<int64_t>(t) * (t + 1) / 2;
    for (int64_t idx = threadIdx.x; idx < count; idx += blockDim.x) {
      // Map idx to (a, c) with a <= c in the trailing t-by-t triangle, column-wise:
      // column cc holds rows 0..cc, offset cc*(cc+1)/2.
      int cc = static_cast<int>((sqrt(8.0 * static_cast<double>(idx) + 1.0) - 1.0) * 0.5);
      while (static_cast<int64_t>(cc + 1) * (cc + 2) / 2 <= idx) ++cc;
      while (static_cast<int64_t>(cc) * (cc + 1) / 2 > idx) --cc;
      const int aa = static_cast<int>(idx - static_cast<int64_t>(cc) * (cc + 1) / 2);
      const int a = j + 1 + aa;
      const int c = j + 1 + cc;
      G[static_cast<int64_t>(c) * ldg + a] -=
          G[static_cast<int64_t>(a) * ldg + j] * G[static_cast<int64_t>(c) * ldg + j];
    }
    __syncthreads();
  }
  // Zero the strict lower triangle.
  for (int64_t idx = threadIdx.x; idx < static_cast<int64_t>(k) * k; idx += blockDim.x) {
    const int r = static_cast<int>(idx % k);
    const int c = static_cast<int>(idx / k);
    if (r > c) G[static_cast<int64_t>(c) * ldg + r] = 0.0;
  }
  if (threadIdx.x == 0 && info) *info = failed;
}

// Blocked left-looking Cholesky (upper, G = R^T R) in one CTA of 32 warps, with
// 32-column panels. For panel J (columns j0..j0+jb):
//   1. G[J, c] -= R[0:j0, J]^T R[0:j0, c] for every c >= j0: one warp per column c,
//      lane r owns row j0+r; R[0:j0, J] sits in shared memory, R[l, c] is a
//      broadcast load. Only the upper triangle of the diagonal block is used.
//   2. warp 0 factors the jb x jb diagonal block in registers/shared memory.
//   3. R[J, c] = R_JJ^{-T} G[J, c] for c >= j0+jb: forward substitution with
//      shuffles, one warp per column.
// Dynamic shared memory: k*32 doubles (panel) + 32*33 doubles (diagonal block).
constexpr int kPotrfNB = 32;

__global__ void __launch_bounds__(1024)
potrf_upper_blocked_kernel(double* G, int k, int64_t ldg, int32_t* info, int64_t batch_stride) {
  // batched: CTA b factors the matrix batch_stride doubles after the previous one
  G += static_cast<int64_t>(blockIdx.x) * batch_stride;
  if (info) info += blockIdx.x;
  extern __shared__ double psm[];
  double* panel = psm;                      // [k][32]: panel[l * 32 + r] = R[l, j0 + r]
  double* diag = psm + static_cast<size_t>(k) * kPotrfNB;  // [32][33]
  __shared__ int failed;
  const int warp = threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  const int nwarps = blockDim.x / 32;
  if (threadIdx.x == 0) failed = 0;
  __syncthreads();
  auto g = [&](int r, int c) -> double& { return G[static_cast<int64_t>(c) * ldg + r]; };
  for (int j0 = 0; j0 < k; j0 += kPotrfNB) {
    const int jb = min(kPotrfNB, k - j0);
    // stage R[0:j0, J] (already final) into shared memory
    for (int idx = threadIdx.x; idx < j0 * kPotrfNB; idx += blockDim.x) {
      const int l = idx / kPotrfNB;
      const int r = idx % kPotrfNB;
      panel[idx] = (r < jb) ? g(l, j0 + r) : 0.0;
    }
    __syncthreads();
    // 1. update the panel row against the finished rows 0..j0-1
    for (int c = j0 + warp; c < k; c += nwarps) {
      if (lane < jb && j0 + lane <= c) {
        double acc = 0.0;
        for (int l = 0; l < j0; ++l) acc = fma(panel[l * kPotrfNB + lane], g(l, c), acc);
        g(j0 + lane, c) -= acc;
      }
    }
    __syncthreads();
    // 2. factor the diagonal block (warp 0, column by column)
    if (warp == 0) {
      for (int c = 0; c < jb; ++c)
        if (lane <= c) diag[lane * 33 + c] = g(j0 + lane, j0 + c);
      __syncwarp();
      for (int j = 0; j < jb; ++j) {
        double d = diag[j * 33 + j];
        const bool bad = !(d > 0.0) || !isfinite(d);
        if (bad) {
          if (lane == 0) failed = j0 + j + 1;
          break;
        }
        const double r = sqrt(d);
        __syncwarp();
        if (lane == j) diag[j * 33 + j] = r;
        if (lane > j && lane < jb) diag[j * 33 + lane] /= r;
        __syncwarp();
        // trailing update of the block's upper triangle: a = lane, columns c >= a
        if (lane > j && lane < jb) {
          const double rja = diag[j * 33 + lane];
          for (int c = lane; c < jb; ++c) diag[lane * 33 + c] -= rja * diag[j * 33 + c];
        }
        __syncwarp();
      }
      __syncwarp();
      if (!failed) {
        for (int c = 0; c < jb; ++c)
          if (lane <= c) g(j0 + lane, j0 + c) = diag[lane * 33 + c];
      }
    }
    __syncthreads();
    if (failed) break;
    // 3. triangular solve for the rest of the panel row: R_JJ^T x = G[J, c]
    for (int c = j0 + jb + warp; c < k; c += nwarps) {
      double x = (lane < jb) ? g(j0 + lane, c) : 0.0;
      for (int i = 0; i < jb; ++i) {
        const double xi = __shfl_sync(0xffffffffu, x, i) / diag[i * 33 + i];
        if (lane == i) x = xi;
        if (lane > i && lane < jb) x -= diag[i * 33 + lane] * xi;
      }
      if (lane < jb) g(j0 + lane, c) = x;
    }
    __syncthreads();
  }
  // zero the strict lower triangle
  for (int64_t idx = threadIdx.x; idx < static_cast<int64_t>(k) * k; idx += blockDim.x) {
    const int r = static_cast<int>(idx % k);
    const int c = static_cast<int>(idx / k);
    if (r > c) g(r, c) = 0.0;
  }
  if (threadIdx.x == 0 && info) *info = failed;
}

// One warp per column c of Rinv: back substitution R x = e_c.
__global__ void trinv_upper_kernel(const double* __restrict__ R, int64_t ldr,
                                   double* __restrict__ Rinv, int64_t ldi, int k,
                                   int64_t batch_stride) {
  R += static_cast<int64_t>(blockIdx.y) * batch_stride;
  Rinv += static_cast<int64_t>(blockIdx.y) * batch_stride;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) / 32;
  const int lane = threadIdx.x % 32;
  if (warp >= k) return;
  const int c = warp;
  double* x = Rinv + static_cast<int64_t>(c) * ldi;
  for (int i = lane; i < k; i += 32) x[i] = 0.0;
  __syncwarp();
  if (lane == 0) x[c] = 1.0 / R[static_cast<int64_t>(c) * ldr + c];
  __syncwarp();
  for (int i = c - 1; i >= 0; --i) {
    double s = 0.0;
    for (int l = i + 1 + lane; l <= c; l += 32) s += R[static_cast<int64_t>(l) * ldr + i] * x[l];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) x[i] = -s / R[static_cast<int64_t>(i) * ldr + i];
    __syncwarp();
  }
}

// Cholesky G = R^T R and R^{-1} of one small SPD matrix (k <= kCholSmallMax) per CTA,
// with the matrix in shared memory, padded to a multiple of 32 with the identity
// (column-major, ld kp + 1 so a row and a column both fall on distinct banks).
//  1. Right-looking factorization, two barriers per pivot: every thread reads the
//     pivot and forms its square root and reciprocal itself, row j is scaled, then
//     the trailing upper triangle is updated (a warp per column).
//  2. Blocked inverse in 32 x 32 blocks: each warp inverts one diagonal block by back
//     substitution (a lane per column, no barrier), then block column J of R^{-1}
//     for J = 1, 2, ...: T_I = sum_{L=I}^{J-1} R^{-1}_IL R_LJ for every I < J, and
//     R^{-1}_IJ = -T_I R^{-1}_JJ (from R^{-1} R = I), two barriers per block column.
// Only G's upper triangle is read; R^{-1} is written with a zero lower triangle, and
// info = j + 1 for a non-positive or non-finite pivot j (R^{-1} is then not written).
constexpr int kCholSmallMax = 128;
constexpr int kCholSmallThreads = 512;
constexpr int kCholBlk = 32;
constexpr int kCholBlkLd = kCholBlk + 1;

__host__ __device__ constexpr int chol_small_pad(int k) { return (k + kCholBlk - 1) / kCholBlk * kCholBlk; }

__global__ void __launch_bounds__(kCholSmallThreads)
chol_inv_small_kernel(const double* __restrict__ G, int k, int64_t ldg, int64_t stride_g,
                      double* __restrict__ Rinv, int64_t ldi, int64_t stride_i,
                      int32_t* __restrict__ info) {
  extern __shared__ double csm[];
  const int kp = chol_small_pad(k);
  const int nb = kp / kCholBlk;
  const int ld = kp + 1;
  double* A = csm;                               // kp x ld
  double* dinv = A + static_cast<size_t>(kp) * ld;  // 1 / R_jj
  double* S = dinv + kp;                         // nb diagonal-block inverses, 32 x 33 each
  double* T = S + nb * kCholBlk * kCholBlkLd;    // nb - 1 (at least 1) products
  G += static_cast<int64_t>(blockIdx.x) * stride_g;
  Rinv += static_cast<int64_t>(blockIdx.x) * stride_i;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  constexpr int kWarps = kCholSmallThreads / 32;
  for (int c = warp; c < kp; c += kWarps)
    for (int r = lane; r <= c; r += 32)
      A[r + c * ld] = (c < k) ? G[r + static_cast<int64_t>(c) * ldg] : (r == c ? 1.0 : 0.0);
  __syncthreads();
  int failed = 0;
  for (int j = 0; j < kp; ++j) {
    const double d = A[j + j * ld];
    if (!(d > 0.0) || !isfinite(d)) {
      failed = j + 1;
      break;
    }
    const double inv = 1.0 / sqrt(d);
    for (int c = j + 1 + tid; c < kp; c += kCholSmallThreads) A[j + c * ld] *= inv;
    if (tid == 0) dinv[j] = inv;
    __syncthreads();
    for (int c = j + 1 + warp; c < kp; c += kWarps) {
      const double rjc = A[j + c * ld];
      for (int a = j + 1 + lane; a <= c; a += 32) A[a + c * ld] -= A[j + a * ld] * rjc;
    }
    __syncthreads();
  }
  if (failed) {
    if (tid == 0 && info) info[blockIdx.x] = failed;
    return;
  }
  // diagonal blocks: warp w, lane c computes column c of (R_ww)^{-1}
  if (warp < nb) {
    const int o = warp * kCholBlk;
    double* Sw = S + warp * kCholBlk * kCholBlkLd;
    const int c = lane;
    Sw[c + c * kCholBlkLd] = dinv[o + c];
    for (int i = c - 1; i >= 0; --i) {
      double acc = 0.0;
      for (int l = i + 1; l <= c; ++l)
        acc = fma(A[(o + i) + (o + l) * ld], Sw[l + c * kCholBlkLd], acc);
      Sw[i + c * kCholBlkLd] = -acc * dinv[o + i];
    }
    for (int i = c + 1; i < kCholBlk; ++i) Sw[i + c * kCholBlkLd] = 0.0;
  }
  __syncthreads();
  for (int J = 1; J < nb; ++J) {
    const int count = J * kCholBlk * kCholBlk;
    for (int e = tid; e < count; e += kCholSmallThreads) {
      const int I = e / (kCholBlk * kCholBlk);
      const int rc = e % (kCholBlk * kCholBlk);
      const int c = rc / kCholBlk, r = rc % kCholBlk;
      const double* SI = S + I * kCholBlk * kCholBlkLd;
      double acc = 0.0;
      for (int m = r; m < kCholBlk; ++m)  // (R_II)^{-1} is upper triangular
        acc = fma(SI[r + m * kCholBlkLd], A[(I * kCholBlk + m) + (J * kCholBlk + c) * ld], acc);
      for (int L = I + 1; L < J; ++L)
        for (int m = 0; m < kCholBlk; ++m)
          acc = fma(A[(I * kCholBlk + r) + (L * kCholBlk + m) * ld],
                    A[(L * kCholBlk + m) + (J * kCholBlk + c) * ld], acc);
      T[I * kCholBlk * kCholBlkLd + r + c * kCholBlkLd] = acc;
    }
    __syncthreads();
    const double* SJ = S + J * kCholBlk * kCholBlkLd;
    for (int e = tid; e < count; e += kCholSmallThreads) {
      const int I = e / (kCholBlk * kCholBlk);
      const int rc = e % (kCholBlk * kCholBlk);
      const int c = rc / kCholBlk, r = rc % kCholBlk;
      const double* TI = T + I * kCholBlk * kCholBlkLd;
      double acc = 0.0;
      for (int m = 0; m <= c; ++m) acc = fma(TI[r + m * kCholBlkLd], SJ[m + c * kCholBlkLd], acc);
      A[(I * kCholBlk + r) + (J * kCholBlk + c) * ld] = -acc;
    }
    __syncthreads();
  }
  for (int c = warp; c < k; c += kWarps) {
    for (int r = lane; r < k; r += 32) {
      double v = 0.0;
      if (r <= c) {
        v = (r / kCholBlk == c / kCholBlk)
                ? S[(c / kCholBlk) * kCholBlk * kCholBlkLd + (r % kCholBlk) +
                    (c % kCholBlk) * kCholBlkLd]
                : A[r + c * ld];
      }
      Rinv[r + static_cast<int64_t>(c) * ldi] = v;
    }
  }
  if (tid == 0 && info) info[blockIdx.x] = 0;
}

__global__ void symmetrize_kernel(double* P, int k, int64_t ldp, int64_t batch_stride) {
  P += static_cast<int64_t>(blockIdx.y) * batch_stride;
  const int64_t idx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= static_cast<int64_t>(k) * k) return;
  const int r = static_cast<int>(idx % k);
  const int c = static_cast<int>(idx / k);
  if (r >= c) return;
  const double a = P[static_cast<int64_t>(c) * ldp + r];
  const double b = P[static_cast<int64_t>(r) * ldp + c];
  const double s = 0.5 * (a + b);
  P[static_cast<int64_t>(c) * ldp + r] = s;
  P[static_cast<int64_t>(r) * ldp + c] = s;
}

}  // namespace

void potrf_upper(double* G, int64_t k, int64_t ldg, int32_t* info, cudaStream_t s) {
  FE_REQUIRE(k >= 0 && k <= 16384 && ldg >= k, "potrf_upper: invalid shape");
  if (k == 0) {
    if (info) FE_CHECK_CUDA(cudaMemsetAsync(info, 0, sizeof(int32_t), s));
    return;
  }
  const size_t smem = (static_cast<size_t>(k) * kPotrfNB + 32 * 33) * sizeof(double);
  if (smem <= 200 * 1024) {
    static bool attr = false;
    if (!attr) {
      FE_CHECK_CUDA(cudaFuncSetAttribute(potrf_upper_blocked_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
      attr = true;
    }
    potrf_upper_blocked_kernel<<<1, 1024, smem, s>>>(G, static_cast<int>(k), ldg, info, 0);
    check_launch("potrf_upper_blocked_kernel");
    return;
  }
  potrf_upper_kernel<<<1, 1024, 0, s>>>(G, static_cast<int>(k), ldg, info);
  check_launch("potrf_upper_kernel");
}

void trinv_upper(const double* R, int64_t ldr, double* Rinv, int64_t ldi, int64_t k,
                 cudaStream_t s) {
  FE_REQUIRE(k >= 0 && ldr >= k && ldi >= k, "trinv_upper: invalid shape");
  if (k == 0) return;
  FE_REQUIRE(R != Rinv, "trinv_upper: in-place inverse is not supported");
  const int64_t threads = k * 32;
  trinv_upper_kernel<<<static_cast<unsigned>((threads + 255) / 256), 256, 0, s>>>(
      R, ldr, Rinv, ldi, static_cast<int>(k), 0);
  check_launch("trinv_upper_kernel");
}

// Batched forms for grouped solves: `count` k x k matrices `stride` doubles apart,
// one info word per matrix.
void potrf_upper_batched(double* G, int64_t k, int64_t ldg, int64_t stride, int64_t count,
                         int32_t* info, cudaStream_t s) {
  FE_REQUIRE(k >= 1 && ldg >= k && count >= 1 && count <= 65535 && stride >= ldg * k,
             "potrf_upper_batched: invalid shape");
  const size_t smem = (static_cast<size_t>(k) * kPotrfNB + 32 * 33) * sizeof(double);
  FE_REQUIRE(smem <= 200 * 1024, "potrf_upper_batched: k too large for the blocked kernel");
  FE_CHECK_CUDA(cudaFuncSetAttribute(potrf_upper_blocked_kernel,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  potrf_upper_blocked_kernel<<<static_cast<unsigned>(count), 1024, smem, s>>>(
      G, static_cast<int>(k), ldg, info, stride);
  check_launch("potrf_upper_blocked_kernel");
}

void trinv_upper_batched(const double* R, int64_t ldr, double* Rinv, int64_t ldi, int64_t k,
                         int64_t stride, int64_t count, cudaStream_t s) {
  FE_REQUIRE(k >= 1 && ldr >= k && ldi >= k && count >= 1 && count <= 65535,
             "trinv_upper_batched: invalid shape");
  const int64_t threads = k * 32;
  dim3 grid(static_cast<unsigned>((threads + 255) / 256), static_cast<unsigned>(count));
  trinv_upper_kernel<<<grid, 256, 0, s>>>(R, ldr, Rinv, ldi, static_cast<int>(k), stride);
  check_launch("trinv_upper_kernel");
}

size_t chol_inv_small_smem(int64_t k) {
  const int64_t kp = chol_small_pad(static_cast<int>(k));
  const int64_t nb = kp / kCholBlk;
  return static_cast<size_t>(kp * (kp + 1) + kp +
                             (nb + std::max<int64_t>(nb - 1, 1)) * kCholBlk * kCholBlkLd) *
         sizeof(double);
}

bool chol_inv_small_fits(int64_t k) { return k >= 1 && k <= kCholSmallMax; }

void chol_inv_upper_batched(const double* G, int64_t k, int64_t ldg, int64_t stride_g,
                            double* Rinv, int64_t ldi, int64_t stride_i, int64_t count,
                            int32_t* info, cudaStream_t s) {
  FE_REQUIRE(chol_inv_small_fits(k) && ldg >= k && ldi >= k && count >= 1 && count <= 65535,
             "chol_inv_upper_batched: invalid shape (k must be in [1, 128])");
  const size_t smem = chol_inv_small_smem(k);
  FE_CHECK_CUDA(cudaFuncSetAttribute(chol_inv_small_kernel,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(chol_inv_small_smem(kCholSmallMax))));
  chol_inv_small_kernel<<<static_cast<unsigned>(count), kCholSmallThreads, smem, s>>>(
      G, static_cast<int>(k), ldg, stride_g, Rinv, ldi, stride_i, info);
  check_launch("chol_inv_small_kernel");
}

void symmetrize_batched(double* P, int64_t k, int64_t ldp, int64_t stride, int64_t count,
                        cudaStream_t s) {
  if (k <= 0 || count <= 0) return;
  const int64_t total = k * k;
  dim3 grid(static_cast<unsigned>((total + 255) / 256), static_cast<unsigned>(count));
  symmetrize_kernel<<<grid, 256, 0, s>>>(P, static_cast<int>(k), ldp, stride);
  check_launch("symmetrize_kernel");
}

// C = alpha op(A) B + beta C for small column-major FP64 matrices (projected
// k-by-k algebra): op(A) = A (m x kk) or A^T (A stored kk x m). 32 x 32 output tiles,
// the kk dimension staged through shared memory in 32-wide slabs.
__global__ void small_gemm_kernel(int trans_a, int m, int n, int kk, double alpha,
                                  const double* __restrict__ A, int64_t lda,
                                  const double* __restrict__ B, int64_t ldb, double beta,
                                  double* __restrict__ C, int64_t ldc) {
  __shared__ double As[32][33];
  __shared__ double Bs[32][33];
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8 threads, 4 rows each
  const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int k0 = 0; k0 < kk; k0 += 32) {
    for (int q = ty; q < 32; q += 8) {
      // As[i][l] = op(A)(r0 + i, k0 + l); Bs[l][j] = B(k0 + l, c0 + j)
      const int i = tx, l = q;
      double a = 0.0;
      if (r0 + i < m && k0 + l < kk)
        a = trans_a ? A[static_cast<int64_t>(r0 + i) * lda + (k0 + l)]
                    : A[static_cast<int64_t>(k0 + l) * lda + (r0 + i)];
      As[i][l] = a;
      double b = 0.0;
      if (k0 + tx < kk && c0 + q < n) b = B[static_cast<int64_t>(c0 + q) * ldb + (k0 + tx)];
      Bs[tx][q] = b;
    }
    __syncthreads();
#pragma unroll 8
    for (int l = 0; l < 32; ++l) {
      const double a = As[tx][l];
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q] = fma(a, Bs[l][ty + 8 * q], acc[q]);
    }
    __syncthreads();
  }
  const int i = r0 + tx;
  if (i >= m) return;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int j = c0 + ty + 8 * q;
    if (j < n) {
      double* c = C + static_cast<int64_t>(j) * ldc + i;
      *c = (beta == 0.0) ? alpha * acc[q] : fma(alpha, acc[q], beta * *c);
    }
  }
}

// d[j] = 1 / sqrt(G[j, j]) (1 where the diagonal is not positive).
__global__ void inv_sqrt_diag_kernel(const double* __restrict__ G, int k, int64_t ldg,
                                     double* __restrict__ d) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= k) return;
  const double g = G[static_cast<int64_t>(j) * ldg + j];
  d[j] = g > 0.0 ? 1.0 / sqrt(g) : 1.0;
}

// M[i, j] *= d[i] * d[j] (cols_scaled) or M[i, j] *= d[i] (rows only).
__global__ void diag_scale_kernel(double* __restrict__ M, int rows, int cols, int64_t ldm,
                                  const double* __restrict__ d, int both) {
  const int64_t idx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= static_cast<int64_t>(rows) * cols) return;
  const int i = static_cast<int>(idx % rows), j = static_cast<int>(idx / rows);
  double* x = M + static_cast<int64_t>(j) * ldm + i;
  *x *= both ? d[i] * d[j] : d[i];
}

// Residual split of an FP64 block for the projected operator of the mixed path's FP64
// cycles: Y32 = float(Y), E32 = float(AY - Y diag(theta)) (row-major blocks).
__global__ void shift_split_kernel(int64_t n, int k, const double* __restrict__ AY, int64_t lday,
                                   const double* __restrict__ Y, int64_t ldy,
                                   const double* __restrict__ theta, float* __restrict__ Y32,
                                   float* __restrict__ E32, int64_t ld32) {
  const int64_t total = n * k;
  for (int64_t idx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; idx < total;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i = idx / k;
    const int j = static_cast<int>(idx % k);
    const double y = Y[i * ldy + j];
    Y32[i * ld32 + j] = static_cast<float>(y);
    E32[i * ld32 + j] = static_cast<float>(AY[i * lday + j] - theta[j] * y);
  }
}

// H[r, c] = G[r, c] theta[c] + H1[r, c] (column-major, leading dimension ld).
__global__ void gram_shift_combine_kernel(int k, int64_t ld, const double* __restrict__ G,
                                          const double* __restrict__ theta,
                                          const double* __restrict__ H1, double* __restrict__ H) {
  const int64_t idx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= static_cast<int64_t>(k) * k) return;
  const int r = static_cast<int>(idx % k), c = static_cast<int>(idx / k);
  const int64_t o = static_cast<int64_t>(c) * ld + r;
  H[o] = fma(G[o], theta[c], H1[o]);
}

void small_gemm(bool trans_a, int64_t m, int64_t n, int64_t kk, double alpha, const double* A,
                int64_t lda, const double* B, int64_t ldb, double beta, double* C, int64_t ldc,
                cudaStream_t s) {
  if (m <= 0 || n <= 0) return;
  dim3 grid(static_cast<unsigned>((m + 31) / 32), static_cast<unsigned>((n + 31) / 32));
  small_gemm_kernel<<<grid, dim3(32, 8), 0, s>>>(trans_a ? 1 : 0, static_cast<int>(m),
                                                 static_cast<int>(n), static_cast<int>(kk), alpha,
                                                 A, lda, B, ldb, beta, C, ldc);
  check_launch("small_gemm_kernel");
}

void inv_sqrt_diag(const double* G, int64_t k, int64_t ldg, double* d, cudaStream_t s) {
  inv_sqrt_diag_kernel<<<static_cast<unsigned>((k + 127) / 128), 128, 0, s>>>(
      G, static_cast<int>(k), ldg, d);
  check_launch("inv_sqrt_diag_kernel");
}

void diag_scale(double* M, int64_t rows, int64_t cols, int64_t ldm, const double* d, bool both,
                cudaStream_t s) {
  const int64_t total = rows * cols;
  if (total <= 0) return;
  diag_scale_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, s>>>(
      M, static_cast<int>(rows), static_cast<int>(cols), ldm, d, both ? 1 : 0);
  check_launch("diag_scale_kernel");
}

void shift_split(int64_t n, int64_t k, const double* AY, int64_t lday, const double* Y,
                 int64_t ldy, const double* theta, float* Y32, float* E32, int64_t ld32,
                 cudaStream_t s) {
  if (n <= 0 || k <= 0) return;
  const int64_t total = n * k;
  const unsigned blocks =
      static_cast<unsigned>(std::min<int64_t>((total + 255) / 256, 8LL * num_sms()));
  shift_split_kernel<<<blocks, 256, 0, s>>>(n, static_cast<int>(k), AY, lday, Y, ldy, theta, Y32,
                                            E32, ld32);
  check_launch("shift_split_kernel");
}

void gram_shift_combine(int64_t k, int64_t ld, const double* G, const double* theta,
                        const double* H1, double* H, cudaStream_t s) {
  if (k <= 0) return;
  const int64_t total = k * k;
  gram_shift_combine_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, s>>>(
      static_cast<int>(k), ld, G, theta, H1, H);
  check_launch("gram_shift_combine_kernel");
}

void symmetrize(double* P, int64_t k, int64_t ldp, cudaStream_t s) {
  FE_REQUIRE(k >= 0 && ldp >= k, "symmetrize: invalid shape");
  if (k == 0) return;
  const int64_t total = k * k;
  symmetrize_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, s>>>(
      P, static_cast<int>(k), ldp, 0);
  check_launch("symmetrize_kernel");
}

template <typename S, typename D>
void convert(const S* src, int64_t lds, D* dst, int64_t ldd, int64_t n, int64_t m, cudaStream_t s);

// ------------------------------------------------------------------ CSR ----
Csr* csr_create(int64_t rows, int64_t cols, int64_t nnz, const int32_t* rowptr,
                const int32_t* colind, const double* values) {
  // validate_csr_matrix_data (src/core/CsrMatrix.cpp:11-39)
  FE_REQUIRE(rows >= 0 && cols >= 0, "CsrMatrixData: dimensions must be nonnegative.");
  FE_REQUIRE(rows < 0x7fffffffLL && cols < 0x7fffffffLL, "CsrMatrixData: dimensions exceed int32.");
  FE_REQUIRE(nnz >= 0 && nnz <= 0x7fffffffLL, "CsrMatrixData: nnz exceeds int32.");
  FE_REQUIRE(rowptr != nullptr, "CsrMatrixData: rowptr size must be rows + 1.");
  FE_REQUIRE(nnz == 0 || (colind && values), "CsrMatrixData: colind and values sizes differ.");
  FE_REQUIRE(rowptr[0] == 0, "CsrMatrixData: rowptr must start at zero.");
  FE_REQUIRE(rowptr[rows] == nnz, "CsrMatrixData: rowptr end must equal nnz.");
  for (int64_t i = 1; i <= rows; ++i) {
    FE_REQUIRE(rowptr[i] >= rowptr[i - 1], "CsrMatrixData: rowptr must be nondecreasing.");
  }
  for (int64_t e = 0; e < nnz; ++e) {
    FE_REQUIRE(colind[e] >= 0 && colind[e] < cols, "CsrMatrixData: column index out of range.");
  }
  auto* A = new Csr();
  A->rows = rows;
  A->cols = cols;
  A->nnz = nnz;
  for (int64_t i = 0; i < rows; ++i)
    A->max_row_nnz = std::max<int64_t>(A->max_row_nnz, rowptr[i + 1] - rowptr[i]);
  FE_CHECK_CUDA(cudaGetDevice(&A->device));
  try {
    FE_CHECK_CUDA(cudaMalloc(&A->rowptr, (rows + 1) * sizeof(int32_t)));
    FE_CHECK_CUDA(cudaMalloc(&A->colind, std::max<int64_t>(nnz, 1) * sizeof(int32_t)));
    FE_CHECK_CUDA(cudaMalloc(&A->val64, std::max<int64_t>(nnz, 1) * sizeof(double)));
    FE_CHECK_CUDA(cudaMalloc(&A->val32, std::max<int64_t>(nnz, 1) * sizeof(float)));
    FE_CHECK_CUDA(cudaMemcpy(A->rowptr, rowptr, (rows + 1) * sizeof(int32_t),
                             cudaMemcpyHostToDevice));
    if (nnz > 0) {
      FE_CHECK_CUDA(cudaMemcpy(A->colind, colind, nnz * sizeof(int32_t), cudaMemcpyHostToDevice));
      FE_CHECK_CUDA(cudaMemcpy(A->val64, values, nnz * sizeof(double), cudaMemcpyHostToDevice));
      // FP32 copy of the values, rounded on the device
      convert<double, float>(A->val64, 1, A->val32, 1, nnz, 1, nullptr);
      FE_CHECK_CUDA(cudaStreamSynchronize(nullptr));
    }
  } catch (...) {
    cudaFree(A->rowptr);
    cudaFree(A->colind);
    cudaFree(A->val64);
    cudaFree(A->val32);
    delete A;
    throw;
  }
  return A;
}

void csr_destroy(Csr* A) {
  if (!A) return;
  cudaFree(A->rowptr);
  cudaFree(A->colind);
  cudaFree(A->val64);
  cudaFree(A->val32);
  delete A;
}

}  // namespace fe

using fe::guarded;

extern "C" const char* fe_version(void) { return "fasteig_b200 0.1.0 (sm_100a)"; }

extern "C" const char* fe_last_error(void) { return fe::g_last_error.c_str(); }

extern "C" int64_t fe_launch_count(void) { return fe::g_launches.load(); }

extern "C" int fe_device_count(int* count) {
  return guarded("fe_device_count", [&] {
    FE_REQUIRE(count, "null count");
    int c = 0;
    cudaError_t e = cudaGetDeviceCount(&c);
    if (e != cudaSuccess) {
      cudaGetLastError();
      c = 0;
    }
    *count = c;
  });
}

extern "C" int fe_csr_create(int64_t rows, int64_t cols, int64_t nnz, const int32_t* rowptr,
                             const int32_t* colind, const double* values, fe_csr_t* out) {
  return guarded("fe_csr_create", [&] {
    FE_REQUIRE(out, "null output handle");
    *out = nullptr;
    fe::Csr* A = fe::csr_create(rows, cols, nnz, rowptr, colind, values);
    auto* h = new fe_csr();
    h->m = *A;
    delete A;  // ownership of the device arrays moves to the handle
    *out = h;
  });
}

extern "C" int fe_csr_destroy(fe_csr_t csr) {
  return guarded("fe_csr_destroy", [&] {
    if (!csr) return;
    auto* A = new fe::Csr(csr->m);
    fe::csr_destroy(A);
    delete csr;
  });
}

extern "C" int fe_csr_info(fe_csr_t csr, int64_t* rows, int64_t* cols, int64_t* nnz) {
  return guarded("fe_csr_info", [&] {
    FE_REQUIRE(csr, "null CSR handle");
    if (rows) *rows = csr->m.rows;
    if (cols) *cols = csr->m.cols;
    if (nnz) *nnz = csr->m.nnz;
  });
}

extern "C" int fe_csr_copy_to_host(fe_csr_t csr, int32_t* rowptr, int32_t* colind,
                                   double* values) {
  return guarded("fe_csr_copy_to_host", [&] {
    FE_REQUIRE(csr && rowptr && (csr->m.nnz == 0 || (colind && values)), "null argument");
    const fe::Csr& A = csr->m;
    FE_CHECK_CUDA(cudaMemcpy(rowptr, A.rowptr, (A.rows + 1) * sizeof(int32_t),
                             cudaMemcpyDeviceToHost));
    if (A.nnz > 0) {
      FE_CHECK_CUDA(cudaMemcpy(colind, A.colind, A.nnz * sizeof(int32_t), cudaMemcpyDeviceToHost));
      FE_CHECK_CUDA(cudaMemcpy(values, A.val64, A.nnz * sizeof(double), cudaMemcpyDeviceToHost));
    }
  });
}

extern "C" int fe_potrf_upper_f64(double* G, int64_t k, int64_t ldg, int32_t* info,
                                  void* stream) {
  return guarded("fe_potrf_upper_f64",
                 [&] { fe::potrf_upper(G, k, ldg, info, fe::as_stream(stream)); });
}

extern "C" int fe_trinv_upper_f64(const double* R, int64_t ldr, double* Rinv, int64_t ldi,
                                  int64_t k, void* stream) {
  return guarded("fe_trinv_upper_f64",
                 [&] { fe::trinv_upper(R, ldr, Rinv, ldi, k, fe::as_stream(stream)); });
}

extern "C" int fe_chol_inv_upper_batched_f64(int32_t count, const double* G, int64_t ldg,
                                             int64_t k, double* Rinv, int64_t ldi,
                                             int32_t* info, void* stream) {
  return guarded("fe_chol_inv_upper_batched_f64", [&] {
    FE_REQUIRE(count >= 0 && (count == 0 || (G && Rinv && info)), "null argument");
    if (count == 0) return;
    fe::chol_inv_upper_batched(G, k, ldg, ldg * k, Rinv, ldi, ldi * k, count, info,
                               fe::as_stream(stream));
  });
}

extern "C" int fe_symmetrize_f64(double* P, int64_t k, int64_t ldp, void* stream) {
  return guarded("fe_symmetrize_f64", [&] { fe::symmetrize(P, k, ldp, fe::as_stream(stream)); });
}
