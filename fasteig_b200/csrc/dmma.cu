// FP64 tensor-core (DMMA) kernels for the two tall-skinny FP64 products of the
// solver: the split-K Gram partials X^T Y and the rotation Y = a X C + b Y.
//
// Replace the same reference calls as the SIMT kernels in blocks.cu
// (src/gpu/CudaMultiVector.cpp transpose_multiply :361-406 and
// right_multiply_active_columns :310-359, both cuBLAS Dgemm). tcgen05 has no
// FP64 kind, so FP64 products on sm_100a go through mma.sync.m8n8k4.f64: one
// warp instruction performs 256 FP64 FMAs from one operand element per lane,
// which cuts the shared-memory and issue traffic of the SIMT 8x8 register tile
// by 4x. Operand tiles are staged through a cp.async ring (8-byte copies, any
// alignment; 16-byte copies when rows and columns allow), so global loads of
// stage t+S-1 overlap the MMAs of stage t.
//
// Fragment layouts of m8n8k4 (PTX ISA, "Matrix Fragments for mma.m8n8k4 with
// .f64"): lane l holds A[l/4][l%4], B[l%4][l/4], and D[l/4][2(l%4)+{0,1}].

#include "fe_common.cuh"

#include <algorithm>
#include <string>

namespace fe {
namespace {

__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// cp.async of `bytes` (8 or 16) with zero fill when !pred (no bytes are read then;
// `src` must still be a valid address, so callers pass the operand's base).
template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem, const void* src, bool pred) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  const int sz = pred ? BYTES : 0;
  if constexpr (BYTES == 16) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(src), "r"(sz)
                 : "memory");
  } else {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(src), "r"(sz)
                 : "memory");
  }
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// ------------------------------------------------------------------ Gram ----
// CTA: 64 x 64 output tile (the 64-column tiles of the SIMT plan), 4 warps in
// 2 x 2, each warp 32 x 32 (4 x 4 m8n8 tiles); 16 rows per stage, 4 stages.
// Shared rows are 72 doubles: a fragment load (4 rows x 8 consecutive doubles)
// then falls into two 128-byte wavefronts, the minimum for 256 bytes.
constexpr int kGT = 64;
constexpr int kGR = 16;
constexpr int kGStages = 4;
constexpr int kGLd = 72;
constexpr int kGThreads = 128;
constexpr size_t kGSmem = size_t(kGStages) * 2 * kGR * kGLd * sizeof(double);

template <int VEC>
__global__ void __launch_bounds__(kGThreads)
gram_dmma_kernel(const double* __restrict__ X, int64_t ldx, const double* __restrict__ Y,
                 int64_t ldy, int64_t n, int k, int m, int64_t rows_per_chunk, int symmetric,
                 double* __restrict__ partial, const int64_t* __restrict__ chunk_rows) {
  if (symmetric && blockIdx.x > blockIdx.y) return;  // lower tiles mirror the upper ones
  extern __shared__ double smem[];
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int wi = (warp & 1) * 32;
  const int wj = (warp >> 1) * 32;
  const int i0 = blockIdx.x * kGT;
  const int j0 = blockIdx.y * kGT;
  // Equal chunks of rows_per_chunk rows, or (grouped Grams) the row range
  // [chunk_rows[2z], chunk_rows[2z+1]) of one problem of a concatenated block.
  const int64_t r_begin =
      chunk_rows ? chunk_rows[2 * blockIdx.z] : static_cast<int64_t>(blockIdx.z) * rows_per_chunk;
  const int64_t r_end =
      chunk_rows ? chunk_rows[2 * blockIdx.z + 1] : min(n, r_begin + rows_per_chunk);
  const int stages = static_cast<int>((r_end - r_begin + kGR - 1) / kGR);

  auto xs = [&](int buf) { return smem + static_cast<size_t>(buf) * 2 * kGR * kGLd; };
  auto ys = [&](int buf) { return xs(buf) + kGR * kGLd; };

  // 16 rows x 64 columns per operand: 1024 / VEC copies over 128 threads.
  auto load = [&](int t, int buf) {
    const int64_t rb = r_begin + static_cast<int64_t>(t) * kGR;
    double* xd = xs(buf);
    double* yd = ys(buf);
#pragma unroll
    for (int e = 0; e < (kGR * kGT) / (VEC * kGThreads); ++e) {
      const int idx = (tid + e * kGThreads) * VEC;
      const int rr = idx / kGT;
      const int cc = idx % kGT;
      const int64_t r = rb + rr;
      const bool rin = r < r_end;
      const bool xin = rin && i0 + cc < k;
      const bool yin = rin && j0 + cc < m;
      cp_async<8 * VEC>(xd + rr * kGLd + cc, xin ? X + r * ldx + i0 + cc : X, xin);
      cp_async<8 * VEC>(yd + rr * kGLd + cc, yin ? Y + r * ldy + j0 + cc : Y, yin);
    }
  };

  double acc[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;

#pragma unroll
  for (int t = 0; t < kGStages - 1; ++t) {
    if (t < stages) load(t, t);
    cp_async_commit();
  }
  const int fr = lane & 3;   // row of the slab inside a k4 step
  const int fc = lane >> 2;  // column inside an 8-wide tile
  for (int t = 0; t < stages; ++t) {
    cp_async_wait<kGStages - 2>();
    __syncthreads();
    if (t + kGStages - 1 < stages) load(t + kGStages - 1, (t + kGStages - 1) % kGStages);
    cp_async_commit();
    const double* xd = xs(t % kGStages);
    const double* yd = ys(t % kGStages);
#pragma unroll
    for (int s4 = 0; s4 < kGR / 4; ++s4) {
      double av[4], bv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) av[a] = xd[(s4 * 4 + fr) * kGLd + wi + a * 8 + fc];
#pragma unroll
      for (int b = 0; b < 4; ++b) bv[b] = yd[(s4 * 4 + fr) * kGLd + wj + b * 8 + fc];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) dmma(acc[a][b], av[a], bv[b]);
    }
  }
  cp_async_wait<0>();

  // Partial layout [chunk][j][i] (column-major k x m per chunk).
  double* out = partial + static_cast<int64_t>(blockIdx.z) * k * m;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int i = i0 + wi + a * 8 + fc;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const int j = j0 + wj + b * 8 + 2 * fr + c;
        if (i < k && j < m) out[static_cast<int64_t>(j) * k + i] = acc[a][b][c];
      }
    }
  }
}

// -------------------------------------------------------------- Rotation ----
// CTA: 128 rows x 64 output columns, 8 warps in 4 x 2, each warp 32 x 32; the
// inner dimension advances 16 per stage through a 3-stage ring. X rows are
// staged 20 doubles apart (fragment: 8 rows x 4 doubles -> two wavefronts),
// C rows 72 apart (4 rows x 8 doubles).
constexpr int kRRows = kRotateRowTile;
constexpr int kRCols = 64;
constexpr int kRK = 16;
constexpr int kRStages = 3;
constexpr int kRXLd = 20;
constexpr int kRCLd = 72;
constexpr int kRThreads = 256;
constexpr size_t kRStage = size_t(kRRows) * kRXLd + size_t(kRK) * kRCLd;
constexpr size_t kRSmem = kRStages * kRStage * sizeof(double);

template <int VEC>
__global__ void __launch_bounds__(kRThreads)
rotate_dmma_kernel(const double* __restrict__ X, int64_t ldx, const double* __restrict__ C,
                   int64_t ldc, double* __restrict__ Y, int64_t ldy, int64_t n, int k, int m,
                   double alpha, double beta, int use_beta, int upper_tri,
                   const int32_t* __restrict__ tile_member, int64_t c_stride) {
  // Grouped rotation: row tile t of a concatenated block belongs to problem
  // tile_member[t], whose coefficient matrix starts c_stride doubles further per problem.
  if (tile_member) C += static_cast<int64_t>(tile_member[blockIdx.y]) * c_stride;
  extern __shared__ double smem[];
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int wr = (warp & 3) * 32;
  const int wc = (warp >> 2) * 32;
  const int j0 = blockIdx.x * kRCols;
  const int64_t r0 = static_cast<int64_t>(blockIdx.y) * kRRows;
  // Upper-triangular C (CholQR's R^-1): rows k >= j0 + kRCols are zero for this
  // tile's columns, so those stages are skipped.
  const int k_eff = upper_tri ? min(k, j0 + kRCols) : k;
  const int stages = (k_eff + kRK - 1) / kRK;

  auto xs = [&](int buf) { return smem + static_cast<size_t>(buf) * kRStage; };
  auto cs = [&](int buf) { return xs(buf) + kRRows * kRXLd; };

  auto load = [&](int t, int buf) {
    const int kb = t * kRK;
    double* xd = xs(buf);
    double* cd = cs(buf);
    // X: 128 rows x 16 inner (VEC consecutive inner elements per copy).
#pragma unroll
    for (int e = 0; e < (kRRows * kRK) / (VEC * kRThreads); ++e) {
      const int idx = (tid + e * kRThreads) * VEC;
      const int rr = idx / kRK;
      const int kk = idx % kRK;
      const int64_t r = r0 + rr;
      const bool in = r < n && kb + kk < k;
      cp_async<8 * VEC>(xd + rr * kRXLd + kk, in ? X + r * ldx + kb + kk : X, in);
    }
    // C (column-major): 16 inner x 64 columns, one double per copy (the smem
    // tile is transposed relative to the source).
#pragma unroll
    for (int e = 0; e < (kRK * kRCols) / kRThreads; ++e) {
      const int idx = tid + e * kRThreads;
      const int jj = idx / kRK;
      const int kk = idx % kRK;
      const bool in = kb + kk < k && j0 + jj < m;
      cp_async<8>(cd + kk * kRCLd + jj, in ? C + static_cast<int64_t>(j0 + jj) * ldc + kb + kk : C,
                  in);
    }
  };

  double acc[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;

#pragma unroll
  for (int t = 0; t < kRStages - 1; ++t) {
    if (t < stages) load(t, t);
    cp_async_commit();
  }
  const int fq = lane & 3;
  const int fp = lane >> 2;
  for (int t = 0; t < stages; ++t) {
    cp_async_wait<kRStages - 2>();
    __syncthreads();
    if (t + kRStages - 1 < stages) load(t + kRStages - 1, (t + kRStages - 1) % kRStages);
    cp_async_commit();
    const double* xd = xs(t % kRStages);
    const double* cd = cs(t % kRStages);
#pragma unroll
    for (int s4 = 0; s4 < kRK / 4; ++s4) {
      double av[4], bv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) av[a] = xd[(wr + a * 8 + fp) * kRXLd + s4 * 4 + fq];
#pragma unroll
      for (int b = 0; b < 4; ++b) bv[b] = cd[(s4 * 4 + fq) * kRCLd + wc + b * 8 + fp];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) dmma(acc[a][b], av[a], bv[b]);
    }
  }
  cp_async_wait<0>();

#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int64_t r = r0 + wr + a * 8 + fp;
    if (r >= n) continue;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const int j = j0 + wc + b * 8 + 2 * fq + c;
        if (j < m) {
          double* y = Y + r * ldy + j;
          double v = alpha * acc[a][b][c];
          if (use_beta) v = fma(beta, *y, v);
          *y = v;
        }
      }
    }
  }
}

}  // namespace

// Gram partials on the 64 x 64 tile grid of (tiles_k, tiles_m, chunks). With
// `symmetric` (X and Y the same view) only tiles on and above the diagonal are
// written; the reduction mirrors the rest.
void gram_partial_dmma(const double* X, int64_t ldx, const double* Y, int64_t ldy, int64_t n,
                       int k, int m, int tiles_k, int tiles_m, int chunks, int64_t rows_per_chunk,
                       bool symmetric, double* partial, cudaStream_t s) {
  const bool vec2 = aligned16(X) && aligned16(Y) && ldx % 2 == 0 && ldy % 2 == 0 && k % 2 == 0 &&
                    m % 2 == 0;
  dim3 grid(tiles_k, tiles_m, chunks);
  // The attribute is per function and device; setting it is a cheap host call.
  auto kern = vec2 ? gram_dmma_kernel<2> : gram_dmma_kernel<1>;
  FE_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kGSmem));
  kern<<<grid, kGThreads, kGSmem, s>>>(X, ldx, Y, ldy, n, k, m, rows_per_chunk, symmetric ? 1 : 0,
                                       partial, nullptr);
  check_launch("gram_dmma_kernel");
}

// Grouped Gram partials: chunk z covers rows [chunk_rows[2z], chunk_rows[2z+1]) of
// the concatenated blocks (each chunk inside one problem's rows).
void gram_partial_dmma_ranges(const double* X, int64_t ldx, const double* Y, int64_t ldy, int k,
                              int m, int chunks, const int64_t* chunk_rows, bool symmetric,
                              double* partial, cudaStream_t s) {
  const bool vec2 = aligned16(X) && aligned16(Y) && ldx % 2 == 0 && ldy % 2 == 0 && k % 2 == 0 &&
                    m % 2 == 0;
  FE_REQUIRE(chunks >= 1 && chunks <= 65535, "grouped Gram: chunk count out of range");
  dim3 grid((k + kGT - 1) / kGT, (m + kGT - 1) / kGT, chunks);
  auto kern = vec2 ? gram_dmma_kernel<2> : gram_dmma_kernel<1>;
  FE_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kGSmem));
  kern<<<grid, kGThreads, kGSmem, s>>>(X, ldx, Y, ldy, 0, k, m, 0, symmetric ? 1 : 0, partial,
                                       chunk_rows);
  check_launch("gram_dmma_kernel");
}

void rotate_dmma(const double* X, int64_t ldx, const double* C, int64_t ldc, double* Y,
                 int64_t ldy, int64_t n, int64_t k, int64_t m, double alpha, double beta,
                 cudaStream_t s, bool upper_tri, const int32_t* tile_member, int64_t c_stride) {
  const bool vec2 = aligned16(X) && ldx % 2 == 0 && k % 2 == 0;
  const int64_t row_tiles = (n + kRRows - 1) / kRRows;
  const int64_t col_tiles = (m + kRCols - 1) / kRCols;
  FE_REQUIRE(col_tiles <= 65535, "rotate: too many columns");
  auto kern = vec2 ? rotate_dmma_kernel<2> : rotate_dmma_kernel<1>;
  FE_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kRSmem));
  // Column tiles run fastest so the CTAs sharing an X row tile are adjacent (L2 reuse).
  for (int64_t base = 0; base < row_tiles; base += 65535) {
    const int64_t tiles = std::min<int64_t>(65535, row_tiles - base);
    dim3 grid(static_cast<unsigned>(col_tiles), static_cast<unsigned>(tiles));
    const int64_t r_off = base * kRRows;
    kern<<<grid, kRThreads, kRSmem, s>>>(X + r_off * ldx, ldx, C, ldc, Y + r_off * ldy, ldy,
                                         n - r_off, static_cast<int>(k), static_cast<int>(m),
                                         alpha, beta, beta != 0.0 ? 1 : 0, upper_tri ? 1 : 0,
                                         tile_member ? tile_member + base : nullptr, c_stride);
    check_launch("rotate_dmma_kernel");
  }
}

}  // namespace fe
