// Grouped kernels of the batched Krylov-Schur engine: many independent standard
// problems advance their scalar Lanczos expansions in lockstep, one launch per
// step phase for the whole batch.
//
// Replaces, per problem, the per-step sequence of KrylovSubspace::expand
// (src/core/KrylovSubspace.cpp:125-259: SpMV, two-pass classical Gram-Schmidt
// with device coefficients, CudaMultiVector::orthogonalize_active_columns_device_coeffs
// src/gpu/CudaMultiVector.cpp:477-539, norms with a host sync per step) and the
// projected m x m eigensolve of each restart (CudaLanczosWorkspace::compute_snapshot,
// src/gpu/CudaLanczosWorkspace.cpp:135-194), which the reference runs one problem
// per process.
//
// Layout: the problems' rows are concatenated (problem p owns rows
// [row0_p, row0_p + n_p)); the operator is the block-diagonal CSR of all
// problems, so one SpMV advances every problem. Per-problem reductions run over
// fixed chunks of at most kBatchChunkRows rows that never cross a problem
// boundary and are summed in chunk order, so each problem's arithmetic, and its
// result, is the same alone and inside any batch. Per-problem scalars (current
// column, alpha, beta, the projected matrix T) live on the device, so a whole
// Lanczos step needs no host round trip and is captured once as a CUDA graph.

#include "device.hpp"

#include <algorithm>
#include <cfloat>
#include <memory>
#include <string>
#include <vector>

namespace fe {
namespace {

constexpr int kBT = 256;  // threads per CTA (8 warps)
constexpr int kLaneCols = kBatchMaxDim / 32;

__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < kBT / 32; ++w) s += red[w];
  return s;  // valid in thread 0
}

// part[c] = sum of x^2 over chunk c.
__global__ void __launch_bounds__(kBT) bks_sumsq_kernel(BatchLayout L, const double* __restrict__ x,
                                                        double* __restrict__ part) {
  __shared__ double red[kBT / 32];
  const int c = blockIdx.x;
  const int64_t r0 = L.c_row0[c];
  const int rows = L.c_rows[c];
  double acc = 0.0;
  for (int i = threadIdx.x; i < rows; i += kBT) {
    const double v = x[r0 + i];
    acc = fma(v, v, acc);
  }
  const double s = block_sum(acc, red);
  if (threadIdx.x == 0) part[c] = s;
}

// Start of a Lanczos step: beta = ||f||, 1/beta; breakdown and non-finite norms
// stop the problem (status 2 / 3).
__global__ void bks_begin_kernel(BatchLayout L, BatchState S) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= L.num_problems || !S.active[p]) return;
  double s = 0.0;
  for (int c = L.p_chunk0[p]; c < L.p_chunk0[p] + L.p_nchunks[p]; ++c) s += S.part1[c];
  const double b = sqrt(s);
  if (!isfinite(b) || !(b > DBL_EPSILON)) {
    S.status[p] = isfinite(b) ? 2 : 3;
    S.active[p] = 0;
    return;
  }
  S.beta[p] = b;
  S.inv[p] = 1.0 / b;
}

// q = f / beta and V[:, col] = q for active problems (q = 0 elsewhere).
__global__ void __launch_bounds__(kBT) bks_store_kernel(BatchLayout L, BatchState S,
                                                        const double* __restrict__ f,
                                                        double* __restrict__ q,
                                                        double* __restrict__ V, int64_t ldv) {
  const int c = blockIdx.x;
  const int p = L.c_prob[c];
  const bool act = S.active[p] != 0;
  const double iv = act ? S.inv[p] : 0.0;
  const int j = act ? S.col[p] : 0;
  const int64_t r0 = L.c_row0[c];
  const int rows = L.c_rows[c];
  for (int i = threadIdx.x; i < rows; i += kBT) {
    const int64_t r = r0 + i;
    const double v = act ? f[r] * iv : 0.0;
    q[r] = v;
    if (act) V[r * ldv + j] = v;
  }
}

// w = A q on the rows of active problems only (one thread per row, the block-diagonal
// CSR's global column indices); chunks of finished or waiting problems exit at once.
__global__ void __launch_bounds__(kBT) bks_spmv_kernel(BatchLayout L, BatchState S,
                                                       const int32_t* __restrict__ rowptr,
                                                       const int32_t* __restrict__ colind,
                                                       const double* __restrict__ val,
                                                       const double* __restrict__ q,
                                                       double* __restrict__ w) {
  const int c = blockIdx.x;
  const int p = L.c_prob[c];
  if (!S.active[p]) return;
  const int64_t r0 = L.c_row0[c];
  const int rows = L.c_rows[c];
  for (int i = threadIdx.x; i < rows; i += kBT) {
    const int64_t r = r0 + i;
    double acc = 0.0;
    for (int32_t e = rowptr[r]; e < rowptr[r + 1]; ++e) acc = fma(val[e], q[colind[e]], acc);
    w[r] = acc;
  }
}

// part[c * M + j] = sum over chunk rows of V[r, j] x[r], j <= col (active problems).
__global__ void __launch_bounds__(kBT) bks_dots_kernel(BatchLayout L, BatchState S,
                                                       const double* __restrict__ V, int64_t ldv,
                                                       const double* __restrict__ x,
                                                       double* __restrict__ part) {
  __shared__ double red[kBT / 32][kBatchMaxDim];
  const int c = blockIdx.x;
  const int p = L.c_prob[c];
  if (!S.active[p]) return;
  const int ncols = S.col[p] + 1;
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int64_t r0 = L.c_row0[c];
  const int rows = L.c_rows[c];
  double acc[kLaneCols];
#pragma unroll
  for (int t = 0; t < kLaneCols; ++t) acc[t] = 0.0;
  for (int i = warp; i < rows; i += kBT / 32) {
    const int64_t r = r0 + i;
    const double xv = x[r];
    const double* vr = V + r * ldv;
#pragma unroll
    for (int t = 0; t < kLaneCols; ++t) {
      const int j = lane + 32 * t;
      if (j < ncols) acc[t] = fma(vr[j], xv, acc[t]);
    }
  }
#pragma unroll
  for (int t = 0; t < kLaneCols; ++t) red[warp][lane + 32 * t] = acc[t];
  __syncthreads();
  for (int j = threadIdx.x; j < ncols; j += kBT) {
    double s = 0.0;
    for (int w = 0; w < kBT / 32; ++w) s += red[w][j];
    part[static_cast<int64_t>(c) * L.M + j] = s;
  }
}

// h[p * M + j] = sum over the problem's chunks (in order) of part[c * M + j].
__global__ void bks_dots_finish_kernel(BatchLayout L, BatchState S, const double* __restrict__ part,
                                       double* __restrict__ h) {
  const int p = blockIdx.x;
  if (!S.active[p]) return;
  const int ncols = S.col[p] + 1;
  for (int j = threadIdx.x; j < ncols; j += blockDim.x) {
    double s = 0.0;
    for (int c = L.p_chunk0[p]; c < L.p_chunk0[p] + L.p_nchunks[p]; ++c)
      s += part[static_cast<int64_t>(c) * L.M + j];
    h[static_cast<int64_t>(p) * L.M + j] = s;
  }
}

// First Gram-Schmidt update fused with the second pass's reduction:
// f[r] = w[r] - V[r, :col+1] h1_p, and part[c * M + j] = sum over chunk rows of V[r, j] f[r].
__global__ void __launch_bounds__(kBT) bks_update_dots_kernel(BatchLayout L, BatchState S,
                                                              const double* __restrict__ V,
                                                              int64_t ldv,
                                                              const double* __restrict__ h,
                                                              const double* __restrict__ src,
                                                              double* __restrict__ dst,
                                                              double* __restrict__ part) {
  __shared__ double red[kBT / 32][kBatchMaxDim];
  const int c = blockIdx.x;
  const int p = L.c_prob[c];
  if (!S.active[p]) return;
  const int ncols = S.col[p] + 1;
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  double hr[kLaneCols], acc[kLaneCols];
#pragma unroll
  for (int t = 0; t < kLaneCols; ++t) {
    const int j = lane + 32 * t;
    hr[t] = j < ncols ? h[static_cast<int64_t>(p) * L.M + j] : 0.0;
    acc[t] = 0.0;
  }
  const int64_t r0 = L.c_row0[c];
  const int rows = L.c_rows[c];
  for (int i = warp; i < rows; i += kBT / 32) {
    const int64_t r = r0 + i;
    const double* vr = V + r * ldv;
    double v[kLaneCols];
    double s = 0.0;
#pragma unroll
    for (int t = 0; t < kLaneCols; ++t) {
      const int j = lane + 32 * t;
      v[t] = j < ncols ? vr[j] : 0.0;
      s = fma(v[t], hr[t], s);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    const double fr = src[r] - s;
    if (lane == 0) dst[r] = fr;
#pragma unroll
    for (int t = 0; t < kLaneCols; ++t) acc[t] = fma(v[t], fr, acc[t]);
  }
#pragma unroll
  for (int t = 0; t < kLaneCols; ++t) red[warp][lane + 32 * t] = acc[t];
  __syncthreads();
  for (int j = threadIdx.x; j < ncols; j += kBT) {
    double sum = 0.0;
    for (int w = 0; w < kBT / 32; ++w) sum += red[w][j];
    part[static_cast<int64_t>(c) * L.M + j] = sum;
  }
}

// Second Gram-Schmidt update fused with the norm: f[r] -= V[r, :col+1] h2_p and
// part1[c] = sum over chunk rows of f[r]^2.
__global__ void __launch_bounds__(kBT) bks_update_sumsq_kernel(BatchLayout L, BatchState S,
                                                               const double* __restrict__ V,
                                                               int64_t ldv,
                                                               const double* __restrict__ h,
                                                               double* __restrict__ f) {
  __shared__ double red[kBT / 32];
  const int c = blockIdx.x;
  const int p = L.c_prob[c];
  if (!S.active[p]) return;
  const int ncols = S.col[p] + 1;
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  double hr[kLaneCols];
#pragma unroll
  for (int t = 0; t < kLaneCols; ++t) {
    const int j = lane + 32 * t;
    hr[t] = j < ncols ? h[static_cast<int64_t>(p) * L.M + j] : 0.0;
  }
  const int64_t r0 = L.c_row0[c];
  const int rows = L.c_rows[c];
  double acc = 0.0;
  for (int i = warp; i < rows; i += kBT / 32) {
    const int64_t r = r0 + i;
    const double* vr = V + r * ldv;
    double s = 0.0;
#pragma unroll
    for (int t = 0; t < kLaneCols; ++t) {
      const int j = lane + 32 * t;
      if (j < ncols) s = fma(vr[j], hr[t], s);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    const double fr = f[r] - s;
    if (lane == 0) {
      f[r] = fr;
      acc = fma(fr, fr, acc);
    }
  }
  if (lane == 0) red[warp] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double sum = 0.0;
    for (int w = 0; w < kBT / 32; ++w) sum += red[w];
    S.part1[c] = sum;
  }
}

// End of a Lanczos step: alpha = h1[col] + h2[col], beta_next = ||f||, T updates
// (KrylovSubspace::expand's recording, src/core/KrylovSubspace.cpp:212-247), col++.
__global__ void bks_end_kernel(BatchLayout L, BatchState S) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= L.num_problems || !S.active[p]) return;
  double s = 0.0;
  for (int c = L.p_chunk0[p]; c < L.p_chunk0[p] + L.p_nchunks[p]; ++c) s += S.part1[c];
  const double bn = sqrt(s);
  if (!isfinite(bn)) {
    S.status[p] = 3;
    S.active[p] = 0;
    return;
  }
  const int64_t M = L.M;
  const int j = S.col[p];
  const double alpha = S.h1[p * M + j] + S.h2[p * M + j];
  double* T = S.T + static_cast<int64_t>(p) * M * M;
  if (j != 0 && j != S.restart_row[p]) {
    T[j + (j - 1) * M] = S.beta[p];
    T[(j - 1) + j * M] = S.beta[p];
  }
  T[j + j * M] = alpha;
  if (j == S.restart_row[p]) S.restart_row[p] = -1;
  S.beta_next[p] = bn;
  S.col[p] = j + 1;
  if (j + 1 >= S.mdim[p]) S.active[p] = 0;
}

// Batched symmetric eigensolver for the projected matrices: one CTA per problem,
// parallel cyclic Jacobi (round-robin pairing, m/2 disjoint rotations per round),
// eigenvalues ascending with eigenvectors (W: P x M, Z: P x M x M column-major).
__global__ void __launch_bounds__(kBT) bks_jacobi_kernel(BatchLayout L, const double* __restrict__ T,
                                                         const int32_t* __restrict__ mdim,
                                                         const int32_t* __restrict__ todo,
                                                         double* __restrict__ W,
                                                         double* __restrict__ Z,
                                                         double* __restrict__ Zlast) {
  extern __shared__ double sh[];
  const int p = blockIdx.x;
  if (!todo[p]) return;
  const int m = mdim[p];
  const int ld = m + 1;
  double* A = sh;
  double* Q = sh + m * ld;
  double* cs = Q + m * ld;                       // kBatchMaxDim / 2
  double* sn = cs + kBatchMaxDim / 2;            // kBatchMaxDim / 2
  int* pp = reinterpret_cast<int*>(sn + kBatchMaxDim / 2);
  int* qq = pp + kBatchMaxDim / 2;
  __shared__ double red[kBT / 32];
  __shared__ int done;
  const int64_t M = L.M;
  const double* Tp = T + p * M * M;
  for (int e = threadIdx.x; e < m * m; e += kBT) {
    const int i = e % m, j = e / m;
    A[i + j * ld] = Tp[i + j * M];
    Q[i + j * ld] = i == j ? 1.0 : 0.0;
  }
  __syncthreads();
  const int mm = m + (m & 1);
  for (int sweep = 0; sweep < 40; ++sweep) {
    double off = 0.0, dg = 0.0;
    for (int e = threadIdx.x; e < m * m; e += kBT) {
      const int i = e % m, j = e / m;
      const double a = A[i + j * ld];
      if (i == j) dg = fma(a, a, dg);
      else off = fma(a, a, off);
    }
    const double off_s = block_sum(off, red);
    __syncthreads();
    const double dg_s = block_sum(dg, red);
    if (threadIdx.x == 0) done = !(off_s > 1e-30 * fmax(dg_s, 1e-300));
    __syncthreads();
    if (done) break;
    for (int round = 0; round < mm - 1; ++round) {
      for (int k = threadIdx.x; k < mm / 2; k += kBT) {
        int a, b;
        if (k == 0) {
          a = round;
          b = mm - 1;
        } else {
          a = (round + k) % (mm - 1);
          b = (round - k + (mm - 1)) % (mm - 1);
        }
        const int lo = min(a, b), hi = max(a, b);
        double c = 1.0, s = 0.0;
        if (hi < m) {
          const double apq = A[lo + hi * ld];
          if (apq != 0.0) {
            const double theta = (A[hi + hi * ld] - A[lo + lo * ld]) / (2.0 * apq);
            const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
            c = 1.0 / sqrt(t * t + 1.0);
            s = t * c;
          }
        }
        cs[k] = c;
        sn[k] = s;
        pp[k] = lo;
        qq[k] = hi < m ? hi : lo;
      }
      __syncthreads();
      // columns: A <- A J, Q <- Q J
      for (int e = threadIdx.x; e < (mm / 2) * m; e += kBT) {
        const int k = e / m, i = e % m;
        const double c = cs[k], s = sn[k];
        if (s == 0.0 && c == 1.0) continue;
        const int a = pp[k], b = qq[k];
        const double x = A[i + a * ld], y = A[i + b * ld];
        A[i + a * ld] = c * x - s * y;
        A[i + b * ld] = s * x + c * y;
        const double u = Q[i + a * ld], v = Q[i + b * ld];
        Q[i + a * ld] = c * u - s * v;
        Q[i + b * ld] = s * u + c * v;
      }
      __syncthreads();
      // rows: A <- J^T A
      for (int e = threadIdx.x; e < (mm / 2) * m; e += kBT) {
        const int k = e / m, j = e % m;
        const double c = cs[k], s = sn[k];
        if (s == 0.0 && c == 1.0) continue;
        const int a = pp[k], b = qq[k];
        const double x = A[a + j * ld], y = A[b + j * ld];
        A[a + j * ld] = c * x - s * y;
        A[b + j * ld] = s * x + c * y;
      }
      __syncthreads();
    }
  }
  // Ascending order (stable by index on ties), as a rank per diagonal entry.
  for (int i = threadIdx.x; i < m; i += kBT) {
    const double di = A[i + i * ld];
    int rank = 0;
    for (int j = 0; j < m; ++j) {
      const double dj = A[j + j * ld];
      if (dj < di || (dj == di && j < i)) ++rank;
    }
    W[p * M + rank] = di;
    Zlast[p * M + rank] = Q[(m - 1) + i * ld];
    for (int r = 0; r < m; ++r) Z[p * M * M + r + static_cast<int64_t>(rank) * M] = Q[r + i * ld];
  }
}

// Restart bookkeeping on the device, one CTA per problem: rotation coefficients
// C_p[:, j] = Z_p[:, idx_p[j]] for j < max(keep, keepY), and for restarting
// problems (keep > 0) the new projected matrix T_p: diag(lam_s[:keep]) with the
// coupling row/column at index keep (CpuLanczosWorkspace::prepare_krylov_schur_restart,
// src/core/LanczosWorkspace.cpp:94-107).
__global__ void __launch_bounds__(kBT) bks_restart_kernel(BatchLayout L,
                                                          const int32_t* __restrict__ mdim,
                                                          const int32_t* __restrict__ idx,
                                                          const int32_t* __restrict__ keep,
                                                          const int32_t* __restrict__ keepY,
                                                          const double* __restrict__ diag,
                                                          const double* __restrict__ coup,
                                                          const double* __restrict__ Z,
                                                          double* __restrict__ C,
                                                          double* __restrict__ T) {
  const int p = blockIdx.x;
  const int kp = keep[p], ky = keepY[p];
  const int kc = max(kp, ky);
  if (kc <= 0) return;
  const int m = mdim[p];
  const int64_t M = L.M;
  const double* Zp = Z + p * M * M;
  double* Cp = C + p * M * M;
  const int32_t* ip = idx + p * M;
  for (int e = threadIdx.x; e < m * kc; e += kBT) {
    const int i = e % m, j = e / m;
    Cp[i + j * M] = Zp[i + static_cast<int64_t>(ip[j]) * M];
  }
  if (kp > 0) {
    double* Tp = T + p * M * M;
    for (int e = threadIdx.x; e < M * M; e += kBT) Tp[e] = 0.0;
    __syncthreads();
    for (int j = threadIdx.x; j < kp; j += kBT) {
      Tp[j + j * M] = diag[p * M + j];
      Tp[kp + j * M] = coup[p * M + j];
      Tp[j + kp * M] = coup[p * M + j];
    }
  }
}

// dst[r, :keep_p] = V[r, :m_p] C_p (C_p column-major, leading dimension M); the row
// is read whole before it is written, so dst may be V.
__global__ void __launch_bounds__(kBT) bks_rotate_kernel(BatchLayout L, const double* V, int64_t ldv,
                                                         const double* __restrict__ C,
                                                         const int32_t* __restrict__ mdim,
                                                         const int32_t* __restrict__ keep,
                                                         double* dst, int64_t ldd) {
  extern __shared__ double Cs[];  // m x keep, row-major (index i * keep + j)
  const int c = blockIdx.x;
  const int p = L.c_prob[c];
  const int kp = keep[p];
  if (kp <= 0) return;
  const int m = mdim[p];
  const int64_t M = L.M;
  for (int e = threadIdx.x; e < m * kp; e += kBT) {
    const int i = e / kp, j = e % kp;
    Cs[e] = C[p * M * M + i + static_cast<int64_t>(j) * M];
  }
  __syncthreads();
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int64_t r0 = L.c_row0[c];
  const int rows = L.c_rows[c];
  for (int ii = warp; ii < rows; ii += kBT / 32) {
    const int64_t r = r0 + ii;
    const double* vr = V + r * ldv;
    double x[kLaneCols], out[kLaneCols];
#pragma unroll
    for (int t = 0; t < kLaneCols; ++t) {
      const int j = lane + 32 * t;
      x[t] = j < m ? vr[j] : 0.0;
      out[t] = 0.0;
    }
#pragma unroll
    for (int t = 0; t < kLaneCols; ++t) {
      for (int l = 0; l < 32; ++l) {
        const int i = 32 * t + l;
        if (i >= m) break;
        const double xi = __shfl_sync(0xffffffffu, x[t], l);
#pragma unroll
        for (int u = 0; u < kLaneCols; ++u) {
          const int j = lane + 32 * u;
          if (j < kp) out[u] = fma(xi, Cs[i * kp + j], out[u]);
        }
      }
    }
    __syncwarp();
#pragma unroll
    for (int u = 0; u < kLaneCols; ++u) {
      const int j = lane + 32 * u;
      if (j < kp) dst[r * ldd + j] = out[u];
    }
  }
}

// Final Ritz residuals: per chunk sums of (AY - l Y)^2 and Y^2 for j < nev_p.
__global__ void __launch_bounds__(kBT) bks_resid_kernel(BatchLayout L, const int32_t* __restrict__ nev,
                                                        const double* __restrict__ AY,
                                                        const double* __restrict__ Y, int64_t ld,
                                                        const double* __restrict__ lam, int ldl,
                                                        double* __restrict__ part) {
  __shared__ double red[2][kBT / 32][kBatchMaxDim];
  const int c = blockIdx.x;
  const int p = L.c_prob[c];
  const int ne = nev[p];
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  double ar[kLaneCols], ay[kLaneCols], lv[kLaneCols];
#pragma unroll
  for (int t = 0; t < kLaneCols; ++t) {
    const int j = lane + 32 * t;
    ar[t] = ay[t] = 0.0;
    lv[t] = j < ne ? lam[static_cast<int64_t>(p) * ldl + j] : 0.0;
  }
  const int64_t r0 = L.c_row0[c];
  const int rows = L.c_rows[c];
  for (int i = warp; i < rows; i += kBT / 32) {
    const int64_t r = r0 + i;
#pragma unroll
    for (int t = 0; t < kLaneCols; ++t) {
      const int j = lane + 32 * t;
      if (j < ne) {
        const double y = Y[r * ld + j];
        const double rv = AY[r * ld + j] - lv[t] * y;
        ar[t] = fma(rv, rv, ar[t]);
        ay[t] = fma(y, y, ay[t]);
      }
    }
  }
#pragma unroll
  for (int t = 0; t < kLaneCols; ++t) {
    red[0][warp][lane + 32 * t] = ar[t];
    red[1][warp][lane + 32 * t] = ay[t];
  }
  __syncthreads();
  for (int j = threadIdx.x; j < ne; j += kBT) {
    double a = 0.0, b = 0.0;
    for (int w = 0; w < kBT / 32; ++w) {
      a += red[0][w][j];
      b += red[1][w][j];
    }
    part[static_cast<int64_t>(c) * 2 * ldl + j] = a;
    part[static_cast<int64_t>(c) * 2 * ldl + ldl + j] = b;
  }
}

__global__ void bks_resid_finish_kernel(BatchLayout L, const int32_t* __restrict__ nev,
                                        const double* __restrict__ part,
                                        const double* __restrict__ lam, int ldl,
                                        double* __restrict__ rel) {
  const int p = blockIdx.x;
  for (int j = threadIdx.x; j < nev[p]; j += blockDim.x) {
    double a = 0.0, b = 0.0;
    for (int c = L.p_chunk0[p]; c < L.p_chunk0[p] + L.p_nchunks[p]; ++c) {
      a += part[static_cast<int64_t>(c) * 2 * ldl + j];
      b += part[static_cast<int64_t>(c) * 2 * ldl + ldl + j];
    }
    const double l = lam[static_cast<int64_t>(p) * ldl + j];
    const double den = (1.0 + fabs(l)) * sqrt(b);
    rel[static_cast<int64_t>(p) * ldl + j] = den > 0.0 ? sqrt(a) / den : sqrt(a);
  }
}

// Block-diagonal CSR assembly: rows of problem p shifted by row0_p, entries by nz0_p.
__global__ void bks_offset_copy_kernel(const int32_t* __restrict__ src, int64_t count, int32_t add,
                                       int32_t* __restrict__ dst) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    dst[i] = src[i] + add;
}

unsigned grid_for(int64_t count) {
  return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((count + 255) / 256, 148 * 8)));
}

}  // namespace

void bks_lanczos_step(const BatchLayout& L, const BatchState& S, const Csr& A, double* V,
                      int64_t ldv, double* f, double* q, double* w, cudaStream_t s) {
  const unsigned pc = static_cast<unsigned>(L.num_chunks);
  const unsigned pp = static_cast<unsigned>((L.num_problems + 127) / 128);
  // part1 holds the chunk sums of f^2 on entry (bks_init_norm or the previous step).
  bks_begin_kernel<<<pp, 128, 0, s>>>(L, S);
  check_launch("bks_begin_kernel");
  bks_store_kernel<<<pc, kBT, 0, s>>>(L, S, f, q, V, ldv);
  check_launch("bks_store_kernel");
  bks_spmv_kernel<<<pc, kBT, 0, s>>>(L, S, A.rowptr, A.colind, A.val64, q, w);
  check_launch("bks_spmv_kernel");
  bks_dots_kernel<<<pc, kBT, 0, s>>>(L, S, V, ldv, w, S.part);
  check_launch("bks_dots_kernel");
  bks_dots_finish_kernel<<<static_cast<unsigned>(L.num_problems), 128, 0, s>>>(L, S, S.part, S.h1);
  check_launch("bks_dots_finish_kernel");
  bks_update_dots_kernel<<<pc, kBT, 0, s>>>(L, S, V, ldv, S.h1, w, f, S.part);
  check_launch("bks_update_dots_kernel");
  bks_dots_finish_kernel<<<static_cast<unsigned>(L.num_problems), 128, 0, s>>>(L, S, S.part, S.h2);
  check_launch("bks_dots_finish_kernel");
  bks_update_sumsq_kernel<<<pc, kBT, 0, s>>>(L, S, V, ldv, S.h2, f);
  check_launch("bks_update_sumsq_kernel");
  bks_end_kernel<<<pp, 128, 0, s>>>(L, S);
  check_launch("bks_end_kernel");
}

void bks_init_norm(const BatchLayout& L, const BatchState& S, const double* f, cudaStream_t s) {
  bks_sumsq_kernel<<<static_cast<unsigned>(L.num_chunks), kBT, 0, s>>>(L, f, S.part1);
  check_launch("bks_sumsq_kernel");
}

size_t bks_jacobi_smem(int m) {
  return (2 * static_cast<size_t>(m) * (m + 1) + kBatchMaxDim) * sizeof(double) +
         kBatchMaxDim * sizeof(int);
}

void bks_jacobi(const BatchLayout& L, const double* T, const int32_t* mdim, const int32_t* todo,
                int max_m, double* W, double* Z, double* Zlast, cudaStream_t s) {
  const size_t smem = bks_jacobi_smem(max_m);
  FE_CHECK_CUDA(cudaFuncSetAttribute(bks_jacobi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(smem)));
  bks_jacobi_kernel<<<static_cast<unsigned>(L.num_problems), kBT, smem, s>>>(L, T, mdim, todo, W, Z,
                                                                          Zlast);
  check_launch("bks_jacobi_kernel");
}

void bks_restart(const BatchLayout& L, const int32_t* mdim, const int32_t* idx,
                 const int32_t* keep, const int32_t* keepY, const double* diag,
                 const double* coup, const double* Z, double* C, double* T, cudaStream_t s) {
  bks_restart_kernel<<<static_cast<unsigned>(L.num_problems), kBT, 0, s>>>(L, mdim, idx, keep, keepY,
                                                                        diag, coup, Z, C, T);
  check_launch("bks_restart_kernel");
}

void bks_rotate(const BatchLayout& L, const double* V, int64_t ldv, const double* C,
                const int32_t* mdim, const int32_t* keep, int max_m, int max_keep, double* dst,
                int64_t ldd, cudaStream_t s) {
  if (max_keep <= 0) return;
  const size_t smem = static_cast<size_t>(max_m) * max_keep * sizeof(double);
  FE_CHECK_CUDA(cudaFuncSetAttribute(bks_rotate_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(std::max<size_t>(smem, 16))));
  bks_rotate_kernel<<<static_cast<unsigned>(L.num_chunks), kBT, smem, s>>>(L, V, ldv, C, mdim, keep,
                                                                        dst, ldd);
  check_launch("bks_rotate_kernel");
}

void bks_residuals(const BatchLayout& L, const int32_t* nev, const double* AY, const double* Y,
                   int64_t ld, const double* lam, int ldl, double* part, double* rel,
                   cudaStream_t s) {
  bks_resid_kernel<<<static_cast<unsigned>(L.num_chunks), kBT, 0, s>>>(L, nev, AY, Y, ld, lam, ldl,
                                                                      part);
  check_launch("bks_resid_kernel");
  bks_resid_finish_kernel<<<static_cast<unsigned>(L.num_problems), 128, 0, s>>>(L, nev, part, lam,
                                                                               ldl, rel);
  check_launch("bks_resid_finish_kernel");
}

void bks_offset_copy(const int32_t* src, int64_t count, int32_t add, int32_t* dst, cudaStream_t s) {
  if (count <= 0) return;
  bks_offset_copy_kernel<<<grid_for(count), 256, 0, s>>>(src, count, add, dst);
  check_launch("bks_offset_copy_kernel");
}

}  // namespace fe

// ---------------------------------------------------------------------------
// C ABI: the batch engine's building blocks on their own.
// ---------------------------------------------------------------------------

// Block-diagonal operator of `count` CSR handles (rows and columns offset by the
// preceding parts): one SpMM over it is a grouped SpMM of all parts.
extern "C" int fe_csr_block_diag(int32_t count, const fe_csr_t* parts, fe_csr_t* out) {
  return fe::guarded("fe_csr_block_diag", [&] {
    FE_REQUIRE(count > 0 && parts && out, "null or empty part list");
    *out = nullptr;
    int64_t rows = 0, cols = 0, nnz = 0, maxnz = 0;
    const int device = parts[0] ? parts[0]->m.device : 0;
    for (int32_t p = 0; p < count; ++p) {
      FE_REQUIRE(parts[p], "null CSR handle in part list");
      FE_REQUIRE(parts[p]->m.device == device, "parts live on different devices");
      rows += parts[p]->m.rows;
      cols += parts[p]->m.cols;
      nnz += parts[p]->m.nnz;
      maxnz = std::max(maxnz, parts[p]->m.max_row_nnz);
    }
    FE_REQUIRE(rows < 0x7fffffffLL && cols < 0x7fffffffLL && nnz <= 0x7fffffffLL,
               "block-diagonal operator exceeds int32 indexing");
    FE_CHECK_CUDA(cudaSetDevice(device));
    auto h = std::make_unique<fe_csr>();
    fe::Csr& A = h->m;
    A.rows = rows;
    A.cols = cols;
    A.nnz = nnz;
    A.device = device;
    A.max_row_nnz = maxnz;
    auto fail = [&] {
      cudaFree(A.rowptr);
      cudaFree(A.colind);
      cudaFree(A.val64);
      cudaFree(A.val32);
    };
    try {
      FE_CHECK_CUDA(cudaMalloc(&A.rowptr, (rows + 1) * sizeof(int32_t)));
      FE_CHECK_CUDA(cudaMalloc(&A.colind, std::max<int64_t>(nnz, 1) * sizeof(int32_t)));
      FE_CHECK_CUDA(cudaMalloc(&A.val64, std::max<int64_t>(nnz, 1) * sizeof(double)));
      FE_CHECK_CUDA(cudaMalloc(&A.val32, std::max<int64_t>(nnz, 1) * sizeof(float)));
      int64_t r0 = 0, c0 = 0, z0 = 0;
      for (int32_t p = 0; p < count; ++p) {
        const fe::Csr& P = parts[p]->m;
        fe::bks_offset_copy(P.rowptr, P.rows, static_cast<int32_t>(z0), A.rowptr + r0, nullptr);
        fe::bks_offset_copy(P.colind, P.nnz, static_cast<int32_t>(c0), A.colind + z0, nullptr);
        if (P.nnz > 0) {
          FE_CHECK_CUDA(cudaMemcpyAsync(A.val64 + z0, P.val64, P.nnz * sizeof(double),
                                        cudaMemcpyDeviceToDevice, nullptr));
          FE_CHECK_CUDA(cudaMemcpyAsync(A.val32 + z0, P.val32, P.nnz * sizeof(float),
                                        cudaMemcpyDeviceToDevice, nullptr));
        }
        r0 += P.rows;
        c0 += P.cols;
        z0 += P.nnz;
      }
      const int32_t last = static_cast<int32_t>(nnz);
      FE_CHECK_CUDA(cudaMemcpy(A.rowptr + rows, &last, sizeof(int32_t), cudaMemcpyHostToDevice));
      FE_CHECK_CUDA(cudaStreamSynchronize(nullptr));
    } catch (...) {
      fail();
      throw;
    }
    *out = h.release();
  });
}

// Batched symmetric eigensolver for small FP64 matrices, sizes m[p] (host array),
// stored column-major with leading dimension lda at A + p*lda*lda on the device.
// Writes ascending eigenvalues to W + p*lda and eigenvectors to Z + p*lda*lda.
// Batches whose matrices are all <= 96 run the parallel cyclic Jacobi kernel (one
// CTA per matrix, in shared memory); larger ones the tridiagonal path of syevd.cu.
extern "C" int fe_syevd_batched_f64(int32_t count, const int32_t* m, const double* A, int64_t lda,
                                    double* W, double* Z, void* stream) {
  return fe::guarded("fe_syevd_batched_f64", [&] {
    FE_REQUIRE(count >= 0 && m, "invalid batch");
    if (count == 0) return;
    FE_REQUIRE(A && W && Z, "null matrix pointer");
    int max_m = 1;
    for (int32_t p = 0; p < count; ++p) {
      FE_REQUIRE(m[p] >= 1 && m[p] <= 8192, "matrix size must be in [1, 8192]");
      FE_REQUIRE(m[p] <= lda, "lda smaller than a matrix size");
      max_m = std::max<int>(max_m, m[p]);
    }
    cudaStream_t s = fe::as_stream(stream);
    if (max_m > fe::kBatchMaxDim) {
      // A is input only: decompose a copy (the tridiagonal path overwrites it).
      const size_t mats = static_cast<size_t>(count) * lda * lda * sizeof(double);
      fe::DeviceBuffer copy(mats), info(static_cast<size_t>(count) * sizeof(int32_t)),
          ws(fe::syevd_workspace_bytes(count, lda));
      FE_CHECK_CUDA(cudaMemcpyAsync(copy.get(), A, mats, cudaMemcpyDeviceToDevice, s));
      fe::syevd_batched(count, m, copy.as<double>(), lda, W, Z, info.as<int32_t>(), ws.get(),
                        ws.bytes(), s);
      FE_CHECK_CUDA(cudaStreamSynchronize(s));
      return;
    }
    void *dm = nullptr, *dtodo = nullptr, *dzl = nullptr;
    FE_CHECK_CUDA(cudaMallocAsync(&dm, count * sizeof(int32_t), s));
    FE_CHECK_CUDA(cudaMallocAsync(&dtodo, count * sizeof(int32_t), s));
    FE_CHECK_CUDA(cudaMallocAsync(&dzl, static_cast<size_t>(count) * lda * sizeof(double), s));
    std::vector<int32_t> ones(count, 1);
    try {
      FE_CHECK_CUDA(cudaMemcpyAsync(dm, m, count * sizeof(int32_t), cudaMemcpyHostToDevice, s));
      FE_CHECK_CUDA(cudaMemcpyAsync(dtodo, ones.data(), count * sizeof(int32_t),
                                    cudaMemcpyHostToDevice, s));
      fe::BatchLayout L;
      L.num_problems = count;
      L.M = lda;
      fe::bks_jacobi(L, A, static_cast<int32_t*>(dm), static_cast<int32_t*>(dtodo), max_m, W, Z,
                     static_cast<double*>(dzl), s);
      FE_CHECK_CUDA(cudaStreamSynchronize(s));
    } catch (...) {
      cudaFreeAsync(dm, s);
      cudaFreeAsync(dtodo, s);
      cudaFreeAsync(dzl, s);
      throw;
    }
    cudaFreeAsync(dm, s);
    cudaFreeAsync(dtodo, s);
    cudaFreeAsync(dzl, s);
  });
}
