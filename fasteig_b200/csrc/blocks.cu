// Dense tall-skinny block kernels: Gram X^T Y, rotation X*C, Ritz residuals
// with column norms, column norms, precision conversion.
//
// Replaces (src/gpu/CudaMultiVector.cpp) transpose_multiply (:361-406: Dgemm
// T,N plus a cudaMalloc/cudaFree and a device-to-host sync per call),
// right_multiply_active_columns (:310-359: cudaMalloc + host-to-device copy of
// C per call, Dgemm N,N), add_scaled_columns (:409-433: one Daxpy per column)
// and column_norms (:435-474: one Dnrm2 per column + sync).
//
// These SIMT kernels are the precise path: Gram products are accumulated in
// FP64 (products of FP32 inputs are exact in FP64), split over row chunks whose
// partial Grams are reduced in a fixed order, so results are deterministic.

#include "fe_common.cuh"

#include <algorithm>
#include <climits>
#include <mutex>
#include <string>
#include <type_traits>

namespace fe {
namespace {

// ---------------------------------------------------------------- Gram ----
constexpr int kGT = 64;    // output tile (k and m)
constexpr int kGK = 32;    // rows per smem stage
constexpr int kGramThreads = 64;      // 8 x 8 threads, 8 x 8 outputs each
// Row chunks are sized for about four waves of resident CTAs (five 2-warp CTAs per
// SM at 190 registers per thread) on 148 SMs, so load latency of one CTA hides
// behind the FMAs of the others.
constexpr int kGramTargetCtas = 148 * 5 * 4;

// 8x8 outputs per thread (rows ty + 8a, columns tx + 8b): 16 shared-memory loads
// feed 64 FP64 FMAs, which matches the FP64 pipe to the shared-memory bandwidth.
template <typename T>
__global__ void __launch_bounds__(kGramThreads)
gram_partial_kernel(const T* __restrict__ X, int64_t ldx, const T* __restrict__ Y, int64_t ldy,
                    int64_t n, int k, int m, int64_t rows_per_chunk,
                    double* __restrict__ partial) {
  __shared__ double Xs[kGK][kGT + 1];
  __shared__ double Ys[kGK][kGT + 1];
  const int tx = threadIdx.x % 8;
  const int ty = threadIdx.x / 8;
  const int i0 = blockIdx.x * kGT;
  const int j0 = blockIdx.y * kGT;
  const int64_t r_begin = static_cast<int64_t>(blockIdx.z) * rows_per_chunk;
  const int64_t r_end = min(n, r_begin + rows_per_chunk);

  double acc[8][8];
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int b = 0; b < 8; ++b) acc[a][b] = 0.0;

  for (int64_t r0 = r_begin; r0 < r_end; r0 += kGK) {
    // 32 rows x 64 columns per operand, 32 elements per thread, coalesced along columns.
#pragma unroll 8
    for (int e = 0; e < (kGK * kGT) / kGramThreads; ++e) {
      const int idx = threadIdx.x + e * kGramThreads;
      const int rr = idx / kGT;
      const int cc = idx % kGT;
      const int64_t r = r0 + rr;
      double xv = 0.0, yv = 0.0;
      if (r < r_end) {
        if (i0 + cc < k) xv = static_cast<double>(X[r * ldx + i0 + cc]);
        if (j0 + cc < m) yv = static_cast<double>(Y[r * ldy + j0 + cc]);
      }
      Xs[rr][cc] = xv;
      Ys[rr][cc] = yv;
    }
    __syncthreads();
#pragma unroll 4
    for (int rr = 0; rr < kGK; ++rr) {
      double xv[8], yv[8];
#pragma unroll
      for (int a = 0; a < 8; ++a) xv[a] = Xs[rr][ty + 8 * a];
#pragma unroll
      for (int b = 0; b < 8; ++b) yv[b] = Ys[rr][tx + 8 * b];
#pragma unroll
      for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < 8; ++b) acc[a][b] = fma(xv[a], yv[b], acc[a][b]);
    }
    __syncthreads();
  }
  double* out = partial + static_cast<int64_t>(blockIdx.z) * k * m;
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const int i = i0 + ty + 8 * a;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const int j = j0 + tx + 8 * b;
      if (i < k && j < m) out[static_cast<int64_t>(j) * k + i] = acc[a][b];
    }
  }
}

// With `symmetric` (k == m, only tiles on and above the diagonal computed) an
// entry below the diagonal tiles reads its mirror (j, i).
__global__ void gram_reduce_kernel(const double* __restrict__ partial, int chunks, int k, int m,
                                   double* __restrict__ G, int64_t ldg, int symmetric) {
  const int64_t idx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t total = static_cast<int64_t>(k) * m;
  if (idx >= total) return;
  const int i = static_cast<int>(idx % k);
  const int j = static_cast<int>(idx / k);
  const int64_t src =
      (symmetric && i / kGT > j / kGT) ? static_cast<int64_t>(i) * k + j : idx;
  double s = 0.0;
  for (int c = 0; c < chunks; ++c) s += partial[static_cast<int64_t>(c) * total + src];
  G[static_cast<int64_t>(j) * ldg + i] = s;
}

struct GramPlan {
  int tiles_k, tiles_m, chunks;
  int64_t rows_per_chunk;
  size_t bytes;
};

// max_chunks caps the number of row chunks (so the partials fit a fixed scratch).
GramPlan gram_plan(int64_t n, int64_t k, int64_t m, int64_t max_chunks = INT32_MAX) {
  GramPlan p{};
  p.tiles_k = static_cast<int>((k + kGT - 1) / kGT);
  p.tiles_m = static_cast<int>((m + kGT - 1) / kGT);
  const int64_t tiles = std::max<int64_t>(1, static_cast<int64_t>(p.tiles_k) * p.tiles_m);
  int64_t chunks = (kGramTargetCtas + tiles - 1) / tiles;
  chunks = std::max<int64_t>(1, std::min<int64_t>(chunks, (n + 255) / 256));
  chunks = std::max<int64_t>(1, std::min<int64_t>(chunks, max_chunks));
  int64_t rpc = (n + chunks - 1) / chunks;
  rpc = ((rpc + kGK - 1) / kGK) * kGK;
  chunks = std::max<int64_t>(1, (n + rpc - 1) / rpc);
  p.chunks = static_cast<int>(chunks);
  p.rows_per_chunk = rpc;
  p.bytes = static_cast<size_t>(chunks) * k * m * sizeof(double);
  return p;
}

// --------------------------------------------------------------- Rotation ----
constexpr int kRT = 64;  // rows and output columns per tile
constexpr int kRK = 32;  // inner (k) stage
constexpr int kRotThreads = 64;  // 8 x 8 threads, 8 x 8 outputs each

template <typename T>
__global__ void __launch_bounds__(kRotThreads)
rotate_kernel(const T* __restrict__ X, int64_t ldx, const double* __restrict__ C, int64_t ldc,
              T* __restrict__ Y, int64_t ldy, int64_t n, int k, int m, T alpha, T beta,
              int use_beta) {
  __shared__ T Xs[kRT][kRK + 1];
  __shared__ T Cs[kRK][kRT + 1];
  const int tx = threadIdx.x % 8;
  const int ty = threadIdx.x / 8;
  const int j0 = blockIdx.x * kRT;
  const int64_t r0 = static_cast<int64_t>(blockIdx.y) * kRT;

  T acc[8][8];
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int b = 0; b < 8; ++b) acc[a][b] = T(0);

  for (int k0 = 0; k0 < k; k0 += kRK) {
#pragma unroll 8
    for (int e = 0; e < (kRT * kRK) / kRotThreads; ++e) {
      const int idx = threadIdx.x + e * kRotThreads;
      // X tile: 64 rows x 32 inner, coalesced along inner index.
      const int rr = idx / kRK;
      const int kk = idx % kRK;
      const int64_t r = r0 + rr;
      Xs[rr][kk] = (r < n && k0 + kk < k) ? X[r * ldx + k0 + kk] : T(0);
      // C tile: 32 inner x 64 columns, column-major source, coalesced along inner.
      const int cj = idx / kRK;
      const int ck = idx % kRK;
      Cs[ck][cj] = (k0 + ck < k && j0 + cj < m)
                       ? static_cast<T>(C[static_cast<int64_t>(j0 + cj) * ldc + k0 + ck])
                       : T(0);
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < kRK; ++kk) {
      T xv[8], cv[8];
#pragma unroll
      for (int a = 0; a < 8; ++a) xv[a] = Xs[ty + 8 * a][kk];
#pragma unroll
      for (int b = 0; b < 8; ++b) cv[b] = Cs[kk][tx + 8 * b];
#pragma unroll
      for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < 8; ++b) acc[a][b] = fma(xv[a], cv[b], acc[a][b]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const int64_t r = r0 + ty + 8 * a;
    if (r >= n) continue;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const int j = j0 + tx + 8 * b;
      if (j < m) {
        T* y = Y + r * ldy + j;
        T v = alpha * acc[a][b];
        if (use_beta) v = fma(beta, *y, v);
        *y = v;
      }
    }
  }
}

// -------------------------------------------------- Residual and norms ----
constexpr int kNormCols = 32;       // columns per CTA (one per lane)
constexpr int kNormTargetChunks = 256;

// R = AX - lambda * MX, per-column sums of squares of R and MX (FP64), per chunk.
template <typename T>
__global__ void __launch_bounds__(256)
residual_partial_kernel(const T* __restrict__ AX, const T* __restrict__ X,
                        const T* __restrict__ BX, int64_t ld, int64_t n, int m,
                        const double* __restrict__ lambda, T* __restrict__ R, int64_t ldr,
                        int64_t rows_per_chunk, double* __restrict__ partial, int mode) {
  // mode 0: norms of X (of BX when given) only; mode 1: residual; mode 2: B-norms
  // sqrt(x . Bx) of the columns of X (BX required).
  __shared__ double red[2][8][kNormCols];
  const int lane = threadIdx.x % 32;
  const int warp = threadIdx.x / 32;
  const int j = blockIdx.x * kNormCols + lane;
  const int64_t r_begin = static_cast<int64_t>(blockIdx.y) * rows_per_chunk;
  const int64_t r_end = min(n, r_begin + rows_per_chunk);
  double sr = 0.0, sx = 0.0;
  if (j < m) {
    const double lam = mode == 1 ? lambda[j] : 0.0;
    const T* M = BX ? BX : X;
    for (int64_t r = r_begin + warp; r < r_end; r += 8) {
      const double mx = static_cast<double>(M[r * ld + j]);
      if (mode == 2) {  // B-inner products x . (Bx)
        sx = fma(static_cast<double>(X[r * ld + j]), mx, sx);
        continue;
      }
      sx = fma(mx, mx, sx);
      if (mode == 1) {
        const T rv = static_cast<T>(static_cast<double>(AX[r * ld + j]) - lam * mx);
        if (R) R[r * ldr + j] = rv;
        const double rd = static_cast<double>(rv);
        sr = fma(rd, rd, sr);
      }
    }
  }
  red[0][warp][lane] = sr;
  red[1][warp][lane] = sx;
  __syncthreads();
  if (warp == 0 && j < m) {
    double a = 0.0, b = 0.0;
    for (int w = 0; w < 8; ++w) {
      a += red[0][w][lane];
      b += red[1][w][lane];
    }
    double* out = partial + static_cast<int64_t>(blockIdx.y) * 2 * m;
    out[j] = a;
    out[m + j] = b;
  }
}

__global__ void residual_finish_kernel(const double* __restrict__ partial, int chunks, int m,
                                       const double* __restrict__ lambda, double* rnorm,
                                       double* xnorm, double* rel, int mode) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  double a = 0.0, b = 0.0;
  for (int c = 0; c < chunks; ++c) {
    a += partial[static_cast<int64_t>(c) * 2 * m + j];
    b += partial[static_cast<int64_t>(c) * 2 * m + m + j];
  }
  const double rn = sqrt(a);
  const double xn = sqrt(fmax(b, 0.0));
  if (mode != 1) {
    xnorm[j] = xn;
    return;
  }
  if (rnorm) rnorm[j] = rn;
  if (xnorm) xnorm[j] = xn;
  if (rel) {
    const double den = (1.0 + fabs(lambda[j])) * xn;
    rel[j] = den > 0.0 ? rn / den : rn;
  }
}

struct NormPlan {
  int col_blocks, chunks;
  int64_t rows_per_chunk;
  size_t bytes;
};

NormPlan norm_plan(int64_t n, int64_t m) {
  NormPlan p{};
  p.col_blocks = static_cast<int>((m + kNormCols - 1) / kNormCols);
  int64_t chunks = std::max<int64_t>(1, kNormTargetChunks / std::max(1, p.col_blocks));
  chunks = std::max<int64_t>(1, std::min<int64_t>(chunks, (n + 63) / 64));
  int64_t rpc = (n + chunks - 1) / chunks;
  p.rows_per_chunk = std::max<int64_t>(1, rpc);
  p.chunks = static_cast<int>((n + p.rows_per_chunk - 1) / p.rows_per_chunk);
  if (p.chunks < 1) p.chunks = 1;
  p.bytes = static_cast<size_t>(p.chunks) * 2 * std::max<int64_t>(m, 1) * sizeof(double);
  return p;
}

template <typename S, typename D>
__global__ void convert_kernel(const S* __restrict__ src, int64_t lds, D* __restrict__ dst,
                               int64_t ldd, int64_t n, int m) {
  const int64_t total = n * m;
  for (int64_t idx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; idx < total;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = idx / m;
    const int c = static_cast<int>(idx % m);
    dst[r * ldd + c] = static_cast<D>(src[r * lds + c]);
  }
}

// ------------------------------------------------ tall-skinny GEMV ----
// The Lanczos recurrences multiply an n x k basis (k up to a few dozen) by one
// vector: y = V^T x and x -= V h. A warp takes a row, its lanes the columns, so
// each basis row is read once, coalesced; partial sums per row chunk are reduced
// in a fixed order (deterministic).
constexpr int kGemvMaxCols = 128;
constexpr int kGemvLaneCols = kGemvMaxCols / 32;
constexpr int kGemvThreads = 256;
constexpr int kGemvTargetChunks = 148 * 8;

template <typename T>
__global__ void __launch_bounds__(kGemvThreads)
gemv_t_partial_kernel(const T* __restrict__ V, int64_t ldv, const T* __restrict__ x, int64_t incx,
                      int64_t n, int k, int64_t rows_per_chunk, double* __restrict__ part) {
  __shared__ double red[kGemvThreads / 32][kGemvMaxCols];
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int64_t r_begin = static_cast<int64_t>(blockIdx.x) * rows_per_chunk;
  const int64_t r_end = min(n, r_begin + rows_per_chunk);
  double acc[kGemvLaneCols];
#pragma unroll
  for (int t = 0; t < kGemvLaneCols; ++t) acc[t] = 0.0;
  for (int64_t r = r_begin + warp; r < r_end; r += kGemvThreads / 32) {
    const double xv = static_cast<double>(x[r * incx]);
    const T* vr = V + r * ldv;
#pragma unroll
    for (int t = 0; t < kGemvLaneCols; ++t) {
      const int j = lane + 32 * t;
      if (j < k) acc[t] = fma(static_cast<double>(vr[j]), xv, acc[t]);
    }
  }
#pragma unroll
  for (int t = 0; t < kGemvLaneCols; ++t) red[warp][lane + 32 * t] = acc[t];
  __syncthreads();
  for (int j = threadIdx.x; j < k; j += kGemvThreads) {
    double sum = 0.0;
    for (int w = 0; w < kGemvThreads / 32; ++w) sum += red[w][j];
    part[static_cast<int64_t>(blockIdx.x) * k + j] = sum;
  }
}

__global__ void gemv_t_reduce_kernel(const double* __restrict__ part, int chunks, int k,
                                     double* __restrict__ y) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= k) return;
  double sum = 0.0;
  for (int c = 0; c < chunks; ++c) sum += part[static_cast<int64_t>(c) * k + j];
  y[j] = sum;
}

template <typename T>
__global__ void __launch_bounds__(kGemvThreads)
gemv_n_kernel(const T* __restrict__ V, int64_t ldv, const double* __restrict__ h, int k,
              T* y, int64_t incy, int64_t n, double alpha, double beta, int use_beta) {
  const int lane = threadIdx.x % 32;
  double hr[kGemvLaneCols];
#pragma unroll
  for (int t = 0; t < kGemvLaneCols; ++t) {
    const int j = lane + 32 * t;
    hr[t] = j < k ? h[j] : 0.0;
  }
  const int64_t warps = static_cast<int64_t>(gridDim.x) * (kGemvThreads / 32);
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * (kGemvThreads / 32) + threadIdx.x / 32;
       r < n; r += warps) {
    const T* vr = V + r * ldv;
    double sum = 0.0;
#pragma unroll
    for (int t = 0; t < kGemvLaneCols; ++t) {
      const int j = lane + 32 * t;
      if (j < k) sum = fma(static_cast<double>(vr[j]), hr[t], sum);
    }
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (lane == 0) {
      T* yr = y + r * incy;
      double v = alpha * sum;
      if (use_beta) v = fma(beta, static_cast<double>(*yr), v);
      *yr = static_cast<T>(v);
    }
  }
}

// Narrow bases (k <= K <= 32, the Lanczos bound estimate and Krylov-Schur bases
// of a few dozen columns): a lane takes a whole row and keeps the K column sums
// in registers, so a warp covers 32 rows per pass instead of one, and the rows'
// loads of a pass are independent. Column sums are reduced across lanes with a
// fixed shuffle tree, then across the CTA's warps in order: deterministic.
template <typename T, int K>
__global__ void __launch_bounds__(kGemvThreads)
gemv_t_rows_kernel(const T* __restrict__ V, int64_t ldv, const T* __restrict__ x, int64_t incx,
                   int64_t n, int k, int64_t rows_per_chunk, double* __restrict__ part) {
  __shared__ double red[kGemvThreads / 32][K];
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int64_t r_begin = static_cast<int64_t>(blockIdx.x) * rows_per_chunk;
  const int64_t r_end = min(n, r_begin + rows_per_chunk);
  double acc[K];
#pragma unroll
  for (int j = 0; j < K; ++j) acc[j] = 0.0;
  for (int64_t r = r_begin + threadIdx.x; r < r_end; r += kGemvThreads) {
    const double xv = static_cast<double>(x[r * incx]);
    const T* vr = V + r * ldv;
#pragma unroll
    for (int j = 0; j < K; ++j)
      if (j < k) acc[j] = fma(static_cast<double>(vr[j]), xv, acc[j]);
  }
#pragma unroll
  for (int j = 0; j < K; ++j) {
    double v = acc[j];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp][j] = v;
  }
  __syncthreads();
  for (int j = threadIdx.x; j < k; j += kGemvThreads) {
    double sum = 0.0;
    for (int w = 0; w < kGemvThreads / 32; ++w) sum += red[w][j];
    part[static_cast<int64_t>(blockIdx.x) * k + j] = sum;
  }
}

// y = alpha * V h + beta * y for narrow V, a lane per row (coalesced y).
template <typename T, int K>
__global__ void __launch_bounds__(kGemvThreads)
gemv_n_rows_kernel(const T* __restrict__ V, int64_t ldv, const double* __restrict__ h, int k,
                   T* y, int64_t incy, int64_t n, double alpha, double beta, int use_beta) {
  double hr[K];
#pragma unroll
  for (int j = 0; j < K; ++j) hr[j] = j < k ? h[j] : 0.0;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * kGemvThreads;
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * kGemvThreads + threadIdx.x; r < n;
       r += stride) {
    const T* vr = V + r * ldv;
    double sum = 0.0;
#pragma unroll
    for (int j = 0; j < K; ++j)
      if (j < k) sum = fma(static_cast<double>(vr[j]), hr[j], sum);
    T* yr = y + r * incy;
    double v = alpha * sum;
    if (use_beta) v = fma(beta, static_cast<double>(*yr), v);
    *yr = static_cast<T>(v);
  }
}

}  // namespace

// Workspace that suffices for every call with n' <= n, k' <= k, m' <= m, so a
// caller can size it once for its largest block: chunks <= target/tiles' + 1 and
// k'*m' <= tiles' * 64 * 64 bound the partial count by (target + tiles) tiles.
size_t gram_workspace_bytes(int64_t n, int64_t k, int64_t m) {
  if (n <= 0 || k <= 0 || m <= 0) return 0;
  const int64_t tiles = ((k + kGT - 1) / kGT) * ((m + kGT - 1) / kGT);
  const int64_t by_tiles = (kGramTargetCtas + tiles) * int64_t(kGT) * kGT;
  const int64_t by_rows = ((n + 255) / 256 + 1) * k * m;
  return static_cast<size_t>(std::min(by_tiles, by_rows)) * sizeof(double);
}

// FP64 products: 0 = DMMA tensor-core kernels (dmma.cu), 1 = SIMT kernels.
static int g_f64_gemm_mode = 0;

void set_f64_gemm_mode(int mode) { g_f64_gemm_mode = mode; }

// Split-K Gram partials for plan p; returns whether only the upper tiles were
// computed (X and Y the same view), which the reduction then mirrors.
template <typename T>
bool launch_gram_partial(const T* X, int64_t ldx, const T* Y, int64_t ldy, int64_t n, int64_t k,
                         int64_t m, const GramPlan& p, double* partial, cudaStream_t s) {
  if constexpr (std::is_same_v<T, double>) {
    if (g_f64_gemm_mode == 0) {
      const bool sym = X == Y && ldx == ldy && k == m;
      gram_partial_dmma(X, ldx, Y, ldy, n, static_cast<int>(k), static_cast<int>(m), p.tiles_k,
                        p.tiles_m, p.chunks, p.rows_per_chunk, sym, partial, s);
      return sym;
    }
  }
  dim3 grid(p.tiles_k, p.tiles_m, p.chunks);
  gram_partial_kernel<T><<<grid, kGramThreads, 0, s>>>(X, ldx, Y, ldy, n, static_cast<int>(k),
                                                       static_cast<int>(m), p.rows_per_chunk,
                                                       partial);
  check_launch("gram_partial_kernel");
  return false;
}

template <typename T>
void gram(const T* X, int64_t ldx, const T* Y, int64_t ldy, int64_t n, int64_t k, int64_t m,
          double* G, int64_t ldg, void* ws, size_t ws_bytes, cudaStream_t s) {
  FE_REQUIRE(n >= 0 && k >= 0 && m >= 0, "gram: negative dimension");
  FE_REQUIRE(k <= 65535 * (int64_t)kGT && m <= 65535 * (int64_t)kGT, "gram: too many columns");
  if (k == 0 || m == 0) return;
  FE_REQUIRE(G && ldg >= k, "gram: invalid output");
  if (n == 0) {
    FE_CHECK_CUDA(cudaMemset2DAsync(G, ldg * sizeof(double), 0, k * sizeof(double), m, s));
    return;
  }
  FE_REQUIRE(X && Y && ldx >= k && ldy >= m, "gram: invalid input block");
  if (m == 1 && k <= kGemvMaxCols) {
    // Basis-times-vector shape (Lanczos): G[:, 0] = X^T y by the GEMV kernels.
    const int64_t chunks =
        std::max<int64_t>(1, std::min<int64_t>(kGemvTargetChunks, (n + 255) / 256));
    const int64_t rpc = (n + chunks - 1) / chunks;
    const int64_t nchunks = (n + rpc - 1) / rpc;
    FE_REQUIRE(ws && ws_bytes >= static_cast<size_t>(nchunks) * k * sizeof(double),
               "gram: workspace too small");
    double* part = static_cast<double*>(ws);
    const int ki = static_cast<int>(k);
    const unsigned grid = static_cast<unsigned>(nchunks);
    if (k <= 8) {
      gemv_t_rows_kernel<T, 8><<<grid, kGemvThreads, 0, s>>>(X, ldx, Y, ldy, n, ki, rpc, part);
    } else if (k <= 16) {
      gemv_t_rows_kernel<T, 16><<<grid, kGemvThreads, 0, s>>>(X, ldx, Y, ldy, n, ki, rpc, part);
    } else if (k <= 32) {
      gemv_t_rows_kernel<T, 32><<<grid, kGemvThreads, 0, s>>>(X, ldx, Y, ldy, n, ki, rpc, part);
    } else {
      gemv_t_partial_kernel<T><<<grid, kGemvThreads, 0, s>>>(X, ldx, Y, ldy, n, ki, rpc, part);
    }
    check_launch("gemv_t_partial_kernel");
    gemv_t_reduce_kernel<<<static_cast<unsigned>((k + 127) / 128), 128, 0, s>>>(
        static_cast<const double*>(ws), static_cast<int>(nchunks), static_cast<int>(k), G);
    check_launch("gemv_t_reduce_kernel");
    return;
  }
  const GramPlan p = gram_plan(n, k, m);
  FE_REQUIRE(ws && ws_bytes >= p.bytes, "gram: workspace too small");
  const bool sym = launch_gram_partial(X, ldx, Y, ldy, n, k, m, p, static_cast<double*>(ws), s);
  const int64_t total = k * m;
  gram_reduce_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, s>>>(
      static_cast<const double*>(ws), p.chunks, static_cast<int>(k), static_cast<int>(m), G, ldg,
      sym ? 1 : 0);
  check_launch("gram_reduce_kernel");
}

template void gram<double>(const double*, int64_t, const double*, int64_t, int64_t, int64_t,
                           int64_t, double*, int64_t, void*, size_t, cudaStream_t);
template void gram<float>(const float*, int64_t, const float*, int64_t, int64_t, int64_t,
                          int64_t, double*, int64_t, void*, size_t, cudaStream_t);

template <typename T>
void rotate(const T* X, int64_t ldx, const double* C, int64_t ldc, T* Y, int64_t ldy, int64_t n,
            int64_t k, int64_t m, double alpha, double beta, cudaStream_t s, bool upper_tri) {
  FE_REQUIRE(n >= 0 && k >= 0 && m >= 0, "rotate: negative dimension");
  if (n == 0 || m == 0) return;
  FE_REQUIRE(Y && ldy >= m, "rotate: invalid output block");
  if (k == 0) {
    // Y = beta * Y (alpha * X * C vanishes).
    FE_REQUIRE(beta == 0.0, "rotate: k == 0 with beta != 0 is not supported");
    FE_CHECK_CUDA(cudaMemset2DAsync(Y, ldy * sizeof(T), 0, m * sizeof(T), n, s));
    return;
  }
  FE_REQUIRE(X && C && ldx >= k && ldc >= k, "rotate: invalid input");
  FE_REQUIRE(!ranges_overlap(X, n, ldx, k, static_cast<const T*>(Y), n, ldy, m),
             "rotate: X and Y overlap");
  if (m == 1 && k <= kGemvMaxCols) {
    // Basis-times-vector shape (Lanczos): y = alpha X c + beta y by the GEMV kernel.
    const int ki = static_cast<int>(k);
    const int ub = beta != 0.0 ? 1 : 0;
    if (k <= 32) {
      const unsigned blocks = static_cast<unsigned>(
          std::max<int64_t>(1, std::min<int64_t>((n + kGemvThreads - 1) / kGemvThreads, 148 * 8)));
      if (k <= 8)
        gemv_n_rows_kernel<T, 8><<<blocks, kGemvThreads, 0, s>>>(X, ldx, C, ki, Y, ldy, n, alpha,
                                                                 beta, ub);
      else if (k <= 16)
        gemv_n_rows_kernel<T, 16><<<blocks, kGemvThreads, 0, s>>>(X, ldx, C, ki, Y, ldy, n, alpha,
                                                                  beta, ub);
      else
        gemv_n_rows_kernel<T, 32><<<blocks, kGemvThreads, 0, s>>>(X, ldx, C, ki, Y, ldy, n, alpha,
                                                                  beta, ub);
    } else {
      const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((n + 7) / 8, 148 * 16));
      gemv_n_kernel<T><<<static_cast<unsigned>(blocks), kGemvThreads, 0, s>>>(
          X, ldx, C, ki, Y, ldy, n, alpha, beta, ub);
    }
    check_launch("gemv_n_kernel");
    return;
  }
  if constexpr (std::is_same_v<T, double>) {
    if (g_f64_gemm_mode == 0) {
      rotate_dmma(X, ldx, C, ldc, Y, ldy, n, k, m, alpha, beta, s, upper_tri);
      return;
    }
  }
  const int64_t row_tiles = (n + kRT - 1) / kRT;
  FE_REQUIRE(row_tiles <= 65535LL * 32768LL, "rotate: too many rows");
  const int64_t col_tiles = (m + kRT - 1) / kRT;
  // Column tiles run fastest so the CTAs sharing an X row tile are adjacent (L2 reuse).
  for (int64_t base = 0; base < row_tiles; base += 65535) {
    const int64_t tiles = std::min<int64_t>(65535, row_tiles - base);
    dim3 grid(static_cast<unsigned>(col_tiles), static_cast<unsigned>(tiles));
    const int64_t r_off = base * kRT;
    rotate_kernel<T><<<grid, kRotThreads, 0, s>>>(X + r_off * ldx, ldx, C, ldc, Y + r_off * ldy, ldy,
                                          n - r_off, static_cast<int>(k), static_cast<int>(m),
                                          T(alpha), T(beta), beta != 0.0 ? 1 : 0);
    check_launch("rotate_kernel");
  }
}

template void rotate<double>(const double*, int64_t, const double*, int64_t, double*, int64_t,
                             int64_t, int64_t, int64_t, double, double, cudaStream_t, bool);
template void rotate<float>(const float*, int64_t, const double*, int64_t, float*, int64_t,
                            int64_t, int64_t, int64_t, double, double, cudaStream_t, bool);

// Bound valid for every call with n' <= n and m' <= m (chunks never exceed the
// target count nor one per 64 rows).
size_t residual_workspace_bytes(int64_t n, int64_t m) {
  if (n <= 0 || m <= 0) return 0;
  const int64_t chunks = std::min<int64_t>(kNormTargetChunks, (n + 63) / 64 + 1);
  return static_cast<size_t>(chunks) * 2 * m * sizeof(double);
}

template <typename T>
void residual_norms(const T* AX, const T* X, const T* BX, int64_t ld, int64_t n, int64_t m,
                    const double* lambda, T* R, int64_t ldr, double* rnorm, double* xnorm,
                    double* rel, void* ws, size_t ws_bytes, cudaStream_t s, int mode) {
  FE_REQUIRE(n >= 0 && m >= 0, "residual_norms: negative dimension");
  if (m == 0) return;
  FE_REQUIRE(X && ld >= m, "residual_norms: invalid block");
  FE_REQUIRE(mode >= 0 && mode <= 2, "residual_norms: invalid mode");
  if (mode == 1) FE_REQUIRE(AX && lambda, "residual_norms: missing AX or lambda");
  if (mode == 2) FE_REQUIRE(BX, "residual_norms: B-norms need BX");
  if (R) FE_REQUIRE(ldr >= m, "residual_norms: invalid R leading dimension");
  FE_REQUIRE(m <= 65535LL * kNormCols, "residual_norms: too many columns");
  const NormPlan p = norm_plan(std::max<int64_t>(n, 1), m);
  FE_REQUIRE(ws && ws_bytes >= p.bytes, "residual_norms: workspace too small");
  if (n == 0) {
    FE_CHECK_CUDA(cudaMemsetAsync(ws, 0, p.bytes, s));
  } else {
    dim3 grid(p.col_blocks, p.chunks);
    residual_partial_kernel<T><<<grid, 256, 0, s>>>(AX, X, BX, ld, n, static_cast<int>(m), lambda,
                                                    R, ldr, p.rows_per_chunk,
                                                    static_cast<double*>(ws), mode);
    check_launch("residual_partial_kernel");
  }
  residual_finish_kernel<<<static_cast<unsigned>((m + 127) / 128), 128, 0, s>>>(
      static_cast<const double*>(ws), n == 0 ? 1 : p.chunks, static_cast<int>(m), lambda, rnorm,
      xnorm, rel, mode);
  check_launch("residual_finish_kernel");
}

template void residual_norms<double>(const double*, const double*, const double*, int64_t,
                                     int64_t, int64_t, const double*, double*, int64_t, double*,
                                     double*, double*, void*, size_t, cudaStream_t, int);
template void residual_norms<float>(const float*, const float*, const float*, int64_t, int64_t,
                                    int64_t, const double*, float*, int64_t, double*, double*,
                                    double*, void*, size_t, cudaStream_t, int);

template <typename S, typename D>
void convert(const S* src, int64_t lds, D* dst, int64_t ldd, int64_t n, int64_t m,
             cudaStream_t s) {
  FE_REQUIRE(n >= 0 && m >= 0 && lds >= m && ldd >= m, "convert: invalid shape");
  if (n == 0 || m == 0) return;
  const int64_t total = n * m;
  const int64_t blocks = std::min<int64_t>((total + 255) / 256, 148 * 32);
  convert_kernel<S, D><<<static_cast<unsigned>(blocks), 256, 0, s>>>(src, lds, dst, ldd, n,
                                                                     static_cast<int>(m));
  check_launch("convert_kernel");
}

template void convert<double, float>(const double*, int64_t, float*, int64_t, int64_t, int64_t,
                                     cudaStream_t);
template void convert<float, double>(const float*, int64_t, double*, int64_t, int64_t, int64_t,
                                     cudaStream_t);
template void convert<double, double>(const double*, int64_t, double*, int64_t, int64_t,
                                      int64_t, cudaStream_t);
template void convert<float, float>(const float*, int64_t, float*, int64_t, int64_t, int64_t,
                                    cudaStream_t);

}  // namespace fe

using fe::guarded;

extern "C" size_t fe_gram_workspace_bytes(int64_t n, int64_t k, int64_t m) {
  return fe::gram_workspace_bytes(n, k, m);
}

extern "C" int fe_gram_f64(const double* X, int64_t ldx, const double* Y, int64_t ldy, int64_t n,
                           int64_t k, int64_t m, double* G, int64_t ldg, void* workspace,
                           size_t workspace_bytes, void* stream) {
  return guarded("fe_gram_f64", [&] {
    fe::gram<double>(X, ldx, Y, ldy, n, k, m, G, ldg, workspace, workspace_bytes,
                     fe::as_stream(stream));
  });
}

extern "C" int fe_gram_f32(const float* X, int64_t ldx, const float* Y, int64_t ldy, int64_t n,
                           int64_t k, int64_t m, double* G, int64_t ldg, void* workspace,
                           size_t workspace_bytes, void* stream) {
  return guarded("fe_gram_f32", [&] {
    fe::gram<float>(X, ldx, Y, ldy, n, k, m, G, ldg, workspace, workspace_bytes,
                    fe::as_stream(stream));
  });
}

extern "C" int fe_rotate_f64(const double* X, int64_t ldx, const double* C, int64_t ldc,
                             double* Y, int64_t ldy, int64_t n, int64_t k, int64_t m,
                             double alpha, double beta, void* stream) {
  return guarded("fe_rotate_f64", [&] {
    fe::rotate<double>(X, ldx, C, ldc, Y, ldy, n, k, m, alpha, beta, fe::as_stream(stream),
                       false);
  });
}

extern "C" int fe_rotate_f32(const float* X, int64_t ldx, const double* C, int64_t ldc, float* Y,
                             int64_t ldy, int64_t n, int64_t k, int64_t m, double alpha,
                             double beta, void* stream) {
  return guarded("fe_rotate_f32", [&] {
    fe::rotate<float>(X, ldx, C, ldc, Y, ldy, n, k, m, alpha, beta, fe::as_stream(stream),
                      false);
  });
}

extern "C" size_t fe_residual_workspace_bytes(int64_t n, int64_t m) {
  return fe::residual_workspace_bytes(n, m);
}

extern "C" int fe_residual_norms_f64(const double* AX, const double* X, const double* BX,
                                     int64_t ld, int64_t n, int64_t m, const double* lambda,
                                     double* R, int64_t ldr, double* rnorm, double* xnorm,
                                     double* rel, void* workspace, size_t workspace_bytes,
                                     void* stream) {
  return guarded("fe_residual_norms_f64", [&] {
    fe::residual_norms<double>(AX, X, BX, ld, n, m, lambda, R, ldr, rnorm, xnorm, rel, workspace,
                               workspace_bytes, fe::as_stream(stream), 1);
  });
}

extern "C" int fe_residual_norms_f32(const float* AX, const float* X, const float* BX,
                                     int64_t ld, int64_t n, int64_t m, const double* lambda,
                                     float* R, int64_t ldr, double* rnorm, double* xnorm,
                                     double* rel, void* workspace, size_t workspace_bytes,
                                     void* stream) {
  return guarded("fe_residual_norms_f32", [&] {
    fe::residual_norms<float>(AX, X, BX, ld, n, m, lambda, R, ldr, rnorm, xnorm, rel, workspace,
                              workspace_bytes, fe::as_stream(stream), 1);
  });
}

extern "C" int fe_column_norms_f64(const double* X, int64_t ld, int64_t n, int64_t m,
                                   double* norms, void* workspace, size_t workspace_bytes,
                                   void* stream) {
  return guarded("fe_column_norms_f64", [&] {
    fe::residual_norms<double>(nullptr, X, nullptr, ld, n, m, nullptr, nullptr, 0, nullptr, norms,
                               nullptr, workspace, workspace_bytes, fe::as_stream(stream), 0);
  });
}

extern "C" int fe_column_norms_f32(const float* X, int64_t ld, int64_t n, int64_t m,
                                   double* norms, void* workspace, size_t workspace_bytes,
                                   void* stream) {
  return guarded("fe_column_norms_f32", [&] {
    fe::residual_norms<float>(nullptr, X, nullptr, ld, n, m, nullptr, nullptr, 0, nullptr, norms,
                              nullptr, workspace, workspace_bytes, fe::as_stream(stream), 0);
  });
}

extern "C" int fe_convert_f64_to_f32(const double* src, int64_t lds, float* dst, int64_t ldd,
                                     int64_t n, int64_t m, void* stream) {
  return guarded("fe_convert_f64_to_f32", [&] {
    fe::convert<double, float>(src, lds, dst, ldd, n, m, fe::as_stream(stream));
  });
}

extern "C" int fe_convert_f32_to_f64(const float* src, int64_t lds, double* dst, int64_t ldd,
                                     int64_t n, int64_t m, void* stream) {
  return guarded("fe_convert_f32_to_f64", [&] {
    fe::convert<float, double>(src, lds, dst, ldd, n, m, fe::as_stream(stream));
  });
}

// ------------------------------------------------------------ vectors ----
namespace fe {
namespace {

// y = a*x + b*y on strided vectors (b == 0 overwrites).
__global__ void vec_axpby_kernel(int64_t n, double a, const double* __restrict__ x, int64_t incx,
                                 double b, double* y, int64_t incy) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double v = a * x[i * incx];
    y[i * incy] = (b == 0.0) ? v : fma(b, y[i * incy], v);
  }
}

// Counter-based uniform(-1,1) fill (splitmix64 of seed and element index).
template <typename T>
__global__ void fill_uniform_kernel(T* X, int64_t ld, int64_t n, int m, uint64_t seed) {
  const int64_t total = n * m;
  for (int64_t idx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; idx < total;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = idx / m;
    const int c = static_cast<int>(idx % m);
    uint64_t z = seed * 0x9E3779B97F4A7C15ull + static_cast<uint64_t>(c) * n + r + 1;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    const double u = static_cast<double>(z >> 11) * (1.0 / 9007199254740992.0);
    X[r * ld + c] = static_cast<T>(2.0 * u - 1.0);
  }
}

}  // namespace

void vec_axpby(int64_t n, double a, const double* x, int64_t incx, double b, double* y,
               int64_t incy, cudaStream_t s) {
  if (n <= 0) return;
  const int64_t blocks = std::min<int64_t>((n + 255) / 256, 148 * 16);
  vec_axpby_kernel<<<static_cast<unsigned>(blocks), 256, 0, s>>>(n, a, x, incx, b, y, incy);
  check_launch("vec_axpby_kernel");
}

// y[i*incy] = x[i] / *nrm with the divisor read on the device (a Lanczos basis
// vector from the residual and its norm, with no host round trip).
__global__ void scale_by_inv_kernel(int64_t n, const double* __restrict__ x,
                                    const double* __restrict__ nrm, double* __restrict__ y,
                                    int64_t incy) {
  const double inv = 1.0 / *nrm;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
    y[i * incy] = x[i] * inv;
}

__global__ void sum2_kernel(const double* a, const double* b, double* out) { *out = *a + *b; }

void scale_by_inv(int64_t n, const double* x, const double* nrm, double* y, int64_t incy,
                  cudaStream_t s) {
  if (n <= 0) return;
  const int64_t blocks = std::min<int64_t>((n + 255) / 256, 148 * 16);
  scale_by_inv_kernel<<<static_cast<unsigned>(blocks), 256, 0, s>>>(n, x, nrm, y, incy);
  check_launch("scale_by_inv_kernel");
}

void sum2(const double* a, const double* b, double* out, cudaStream_t s) {
  sum2_kernel<<<1, 1, 0, s>>>(a, b, out);
  check_launch("sum2_kernel");
}

template <typename T>
void fill_uniform(T* X, int64_t ld, int64_t n, int64_t m, uint64_t seed, cudaStream_t s) {
  if (n <= 0 || m <= 0) return;
  const int64_t blocks = std::min<int64_t>((n * m + 255) / 256, 148 * 32);
  fill_uniform_kernel<T><<<static_cast<unsigned>(blocks), 256, 0, s>>>(X, ld, n,
                                                                       static_cast<int>(m), seed);
  check_launch("fill_uniform_kernel");
}
template void fill_uniform<double>(double*, int64_t, int64_t, int64_t, uint64_t, cudaStream_t);
template void fill_uniform<float>(float*, int64_t, int64_t, int64_t, uint64_t, cudaStream_t);

// ------------------------------------------------- small helper kernels ----
namespace {

// dst[:, j] = src[:, idx[j]] on row-major blocks (column gathers of residuals).
template <typename T>
__global__ void gather_columns_kernel(const T* __restrict__ src, int64_t lds,
                                      const int32_t* __restrict__ idx, int m, T* __restrict__ dst,
                                      int64_t ldd, int64_t n, const double* __restrict__ row_scale) {
  const int64_t total = n * m;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = e / m;
    const int j = static_cast<int>(e % m);
    const T v = src[r * lds + idx[j]];
    dst[r * ldd + j] = row_scale ? static_cast<T>(row_scale[r] * static_cast<double>(v)) : v;
  }
}

// t[r] = 1 / |A_rr| (1 where the diagonal entry is zero or absent): Jacobi.
__global__ void jacobi_kernel(int64_t n, const int32_t* __restrict__ rowptr,
                              const int32_t* __restrict__ colind, const double* __restrict__ val,
                              double* __restrict__ t) {
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double d = 0.0;
    for (int32_t p = rowptr[r]; p < rowptr[r + 1]; ++p)
      if (colind[p] == r) d += val[p];
    d = fabs(d);
    t[r] = d > 0.0 ? 1.0 / d : 1.0;
  }
}

// Column-major small matrices: dst[:, j] = src[:, idx[j]] * (scale ? scale[j] : 1).
__global__ void small_gather_scale_kernel(const double* __restrict__ src, int64_t lds, int rows,
                                          const int32_t* __restrict__ idx,
                                          const double* __restrict__ scale, int m,
                                          double* __restrict__ dst, int64_t ldd) {
  const int64_t total = static_cast<int64_t>(rows) * m;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % rows);
    const int j = static_cast<int>(e / rows);
    const double s = scale ? scale[j] : 1.0;
    dst[static_cast<int64_t>(j) * ldd + i] = src[static_cast<int64_t>(idx[j]) * lds + i] * s;
  }
}

// P[c, r] = P[r, c] for r < rows, c0 <= c < c0 + cols (column-major, ld).
__global__ void mirror_block_kernel(double* P, int64_t ld, int rows, int c0, int cols) {
  const int64_t total = static_cast<int64_t>(rows) * cols;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int r = static_cast<int>(e % rows);
    const int c = c0 + static_cast<int>(e / rows);
    P[static_cast<int64_t>(r) * ld + c] = P[static_cast<int64_t>(c) * ld + r];
  }
}

}  // namespace

template <typename T>
void gather_columns(const T* src, int64_t lds, const int32_t* idx, int64_t m, T* dst, int64_t ldd,
                    int64_t n, cudaStream_t s, const double* row_scale) {
  if (n <= 0 || m <= 0) return;
  const int64_t blocks = std::min<int64_t>((n * m + 255) / 256, 148 * 32);
  gather_columns_kernel<T><<<static_cast<unsigned>(blocks), 256, 0, s>>>(
      src, lds, idx, static_cast<int>(m), dst, ldd, n, row_scale);
  check_launch("gather_columns_kernel");
}
template void gather_columns<double>(const double*, int64_t, const int32_t*, int64_t, double*,
                                     int64_t, int64_t, cudaStream_t, const double*);
template void gather_columns<float>(const float*, int64_t, const int32_t*, int64_t, float*,
                                    int64_t, int64_t, cudaStream_t, const double*);

void jacobi_inverse_diagonal(const Csr& A, double* t, cudaStream_t s) {
  if (A.rows <= 0) return;
  const int64_t blocks = std::min<int64_t>((A.rows + 255) / 256, 148 * 16);
  jacobi_kernel<<<static_cast<unsigned>(blocks), 256, 0, s>>>(A.rows, A.rowptr, A.colind,
                                                             A.val64, t);
  check_launch("jacobi_kernel");
}

void small_gather_scale(const double* src, int64_t lds, int64_t rows, const int32_t* idx,
                        const double* scale, int64_t m, double* dst, int64_t ldd, cudaStream_t s) {
  if (rows <= 0 || m <= 0) return;
  const int64_t blocks = std::min<int64_t>((rows * m + 255) / 256, 1024);
  small_gather_scale_kernel<<<static_cast<unsigned>(blocks), 256, 0, s>>>(
      src, lds, static_cast<int>(rows), idx, scale, static_cast<int>(m), dst, ldd);
  check_launch("small_gather_scale_kernel");
}

namespace {
// Row-major (n x m, ld) -> column-major (n x m, leading dimension n), 32x32 tiles.
__global__ void to_colmajor_kernel(const double* __restrict__ src, int64_t lds, int64_t n, int m,
                                   double* __restrict__ dst) {
  __shared__ double tile[32][33];
  const int64_t r0 = static_cast<int64_t>(blockIdx.x) * 32;
  const int c0 = blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int64_t r = r0 + i;
    const int c = c0 + threadIdx.x;
    tile[i][threadIdx.x] = (r < n && c < m) ? src[r * lds + c] : 0.0;
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int c = c0 + j;
    const int64_t r = r0 + threadIdx.x;
    if (r < n && c < m) dst[static_cast<int64_t>(c) * n + r] = tile[threadIdx.x][j];
  }
}
}  // namespace

void to_colmajor(const double* src, int64_t lds, int64_t n, int64_t m, double* dst,
                 cudaStream_t s) {
  if (n <= 0 || m <= 0) return;
  FE_REQUIRE((n + 31) / 32 <= 0x7fffffffLL && (m + 31) / 32 <= 65535, "to_colmajor: too large");
  dim3 grid(static_cast<unsigned>((n + 31) / 32), static_cast<unsigned>((m + 31) / 32));
  to_colmajor_kernel<<<grid, dim3(32, 8), 0, s>>>(src, lds, n, static_cast<int>(m), dst);
  check_launch("to_colmajor_kernel");
}

void mirror_block(double* P, int64_t ld, int64_t rows, int64_t c0, int64_t cols, cudaStream_t s) {
  if (rows <= 0 || cols <= 0) return;
  const int64_t blocks = std::min<int64_t>((rows * cols + 255) / 256, 1024);
  mirror_block_kernel<<<static_cast<unsigned>(blocks), 256, 0, s>>>(
      P, ld, static_cast<int>(rows), static_cast<int>(c0), static_cast<int>(cols));
  check_launch("mirror_block_kernel");
}

// --------------------------------------------- Gram without any allocation ----
// Some callers cannot allocate device memory when they call us: a host program
// that has already handed all device memory to its own pool, or code on a
// latency-critical path where cudaMalloc (which can synchronize the device) is
// not acceptable and no workspace was set aside. For them the FP64 Gram has a
// variant whose split-K partial sums live in the fixed array below, which every
// GPU that loads this library keeps for the life of the process.
namespace {

constexpr int64_t kStaticGramDoubles = int64_t(1) << 20;  // 8 MiB of FP64 partials
constexpr int kMaxDevices = 64;

__device__ __align__(256) double g_static_gram_scratch[kStaticGramDoubles];

std::mutex g_static_gram_mutex;
double* g_static_gram_ptr[kMaxDevices] = {};

// True when p is still device memory of device dev (false after cudaDeviceReset
// has torn down the context the address came from).
bool device_address_valid(const void* p, int dev) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    (void)cudaGetLastError();  // clear the failed query
    return false;
  }
  return a.type == cudaMemoryTypeDevice && a.device == dev;
}

// Device address of the scratch on the current device. The symbol's name is only
// a host-side stand-in, so the address is looked up once per device (with that
// device current) and cached; a cached address that no longer belongs to the
// device (its context was reset) is looked up again.
double* static_gram_scratch() {
  int dev = 0;
  FE_CHECK_CUDA(cudaGetDevice(&dev));
  FE_REQUIRE(dev >= 0 && dev < kMaxDevices, "static Gram scratch: device index out of range");
  std::lock_guard<std::mutex> lock(g_static_gram_mutex);
  if (!g_static_gram_ptr[dev] || !device_address_valid(g_static_gram_ptr[dev], dev)) {
    void* p = nullptr;
    FE_CHECK_CUDA(cudaGetSymbolAddress(&p, g_static_gram_scratch));
    g_static_gram_ptr[dev] = static_cast<double*>(p);
  }
  return g_static_gram_ptr[dev];
}

}  // namespace

int64_t static_gram_max_entries() { return kStaticGramDoubles; }

void gram_f64_static(const double* X, int64_t ldx, const double* Y, int64_t ldy, int64_t n,
                     int64_t k, int64_t m, double* G, int64_t ldg, cudaStream_t s) {
  FE_REQUIRE(n >= 0 && k >= 0 && m >= 0, "gram: negative dimension");
  FE_REQUIRE(k * m <= kStaticGramDoubles,
             "k*m = " + std::to_string(k * m) + " exceeds the static Gram scratch (k*m <= " +
                 std::to_string(kStaticGramDoubles) + ")");
  FE_REQUIRE(k <= 65535 * (int64_t)kGT && m <= 65535 * (int64_t)kGT, "gram: too many columns");
  if (k == 0 || m == 0) return;
  FE_REQUIRE(G && ldg >= k, "gram: invalid output");
  double* scratch = static_gram_scratch();
  if (n == 0) {
    FE_CHECK_CUDA(cudaMemset2DAsync(G, ldg * sizeof(double), 0, k * sizeof(double), m, s));
    return;
  }
  FE_REQUIRE(X && Y && ldx >= k && ldy >= m, "gram: invalid input block");
  // As many row chunks as the scratch holds (each chunk's k x m partial is written
  // in full by the partial kernel, so nothing needs clearing between calls).
  const GramPlan p = gram_plan(n, k, m, std::max<int64_t>(1, kStaticGramDoubles / (k * m)));
  const bool sym = launch_gram_partial(X, ldx, Y, ldy, n, k, m, p, scratch, s);
  const int64_t total = k * m;
  gram_reduce_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, s>>>(
      scratch, p.chunks, static_cast<int>(k), static_cast<int>(m), G, ldg, sym ? 1 : 0);
  check_launch("gram_reduce_kernel");
}

}  // namespace fe

extern "C" int fe_gram_f64_noalloc(const double* X, int64_t ldx, const double* Y, int64_t ldy,
                                   int64_t n, int64_t k, int64_t m, double* G, int64_t ldg,
                                   void* stream) {
  return fe::guarded("fe_gram_f64_noalloc", [&] {
    fe::gram_f64_static(X, ldx, Y, ldy, n, k, m, G, ldg, fe::as_stream(stream));
  });
}

extern "C" int64_t fe_gram_f64_noalloc_max_entries(void) { return fe::static_gram_max_entries(); }
