// Symmetric eigensolver for small dense FP64 matrices on the device (the projected
// k-by-k problems of Rayleigh-Ritz and Krylov-Schur). It replaces the Dsyevd call
// of the reference's GPU path (src/gpu/CudaLanczosWorkspace.cpp:155-157) and the
// host Eigen SelfAdjointEigenSolver of its CPU path (src/core/RitzExtraction.cpp:104).
//
// Four kernels, each batched over matrices (matrix p: A + p*lda*lda, size m[p]):
//   1. sytrd: Householder tridiagonalization, one cluster of 8 CTAs per matrix while
//      the matrix fits their shared memory (k <= 469), else one CTA. Step j reflects
//      column j below the diagonal (dlarfg convention: beta = -sign(alpha)||x||,
//      tau = (beta - alpha)/beta, v = x/(alpha - beta), v0 = 1), then
//      p = tau A22 v, w = p - (tau/2)(p.v) v, A22 -= v w^T + w v^T (both triangles
//      kept). The trailing matrix moves into shared memory once it fits. The
//      reflectors stay in A's strictly lower part for step 4.
//   2. stebz: every eigenvalue of the tridiagonal by multisection on its Sturm
//      count, one CTA per eigenvalue index (ascending order by construction).
//   3. stein: eigenvectors of the tridiagonal by inverse iteration (LU of T - lambda
//      I with partial pivoting, tiny pivots replaced by eps*||T||, three solves from
//      a hashed start vector), one warp per cluster of eigenvalues closer than
//      1e-4 ||T||; members of a cluster are orthogonalized against the earlier ones
//      (modified Gram-Schmidt) after every solve.
//   4. ormtr: Z = H_0 H_1 ... H_{m-3} Z_T, one warp per column of Z (columns in
//      shared memory, reflectors streamed through it).
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <string>
#include <utility>

#include <cooperative_groups.h>

#include "device.hpp"
#include "fe_common.cuh"

namespace fe {
namespace {

constexpr int kTrdThreads = 1024;
constexpr double kEps = 2.220446049250313e-16;
constexpr double kTiny = 2.2250738585072014e-308;  // smallest normal double
constexpr double kClusterTol = 1e-4;                 // relative to ||T||

__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();  // red may still be read from the previous reduction
  if (lane == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  const int nw = (blockDim.x + 31) >> 5;
  for (int i = 0; i < nw; ++i) t += red[i];
  return t;
}

// Householder tridiagonalization of A (symmetric, both triangles read and kept).
// Dynamic shared memory: v, p/w (2 * kmax doubles), 32 reduction slots, then the
// trailing-matrix tile of up to `tile_cap` doubles.
__global__ void __launch_bounds__(kTrdThreads, 1)
sytrd_kernel(const int32_t* __restrict__ msz, double* __restrict__ A, int64_t lda,
             double* __restrict__ d, double* __restrict__ e, double* __restrict__ tau,
             int64_t vec_stride, int kmax, int64_t tile_cap) {
  extern __shared__ double sh[];
  const int p = blockIdx.x;
  const int k = msz[p];
  double* Ap = A + static_cast<int64_t>(p) * lda * lda;
  double* dp = d + p * vec_stride;
  double* ep = e + p * vec_stride;
  double* tp = tau + p * vec_stride;
  double* v = sh;
  double* w = sh + kmax;
  double* red = sh + 2 * kmax;
  double* tile = red + 32;
  const int tid = threadIdx.x;
  __shared__ double s_scale, s_tau;

  // Working view of the trailing matrix: global memory until it fits the tile.
  double* M = Ap;
  int64_t ldm = lda;
  int64_t moff = 0;  // the view's element (0,0) is A(moff, moff)
  bool in_smem = false;
  for (int j = 0; j + 2 < k; ++j) {
    const int m = k - j - 1;  // rows/cols of A22 = A(j+1:, j+1:)
    if (!in_smem && static_cast<int64_t>(m + 1) * (m + 1) <= tile_cap) {
      // Move A(j:, j:) into shared memory (column-major, ld = m + 1).
      const int mm = m + 1;
      for (int64_t idx = tid; idx < static_cast<int64_t>(mm) * mm; idx += blockDim.x) {
        const int r = static_cast<int>(idx % mm), c = static_cast<int>(idx / mm);
        tile[idx] = Ap[(j + c) * lda + (j + r)];
      }
      __syncthreads();
      M = tile;
      ldm = mm;
      moff = j;
      in_smem = true;
    }
    const int64_t o = j - moff;  // A(j, j) in the view
    // Column j below the diagonal and its norm.
    double part = 0.0;
    for (int i = tid; i < m; i += blockDim.x) {
      const double x = M[o * ldm + (o + 1 + i)];
      v[i] = x;
      if (i > 0) part += x * x;
    }
    const double xn2 = block_sum(part, red);
    if (tid == 0) {
      const double alpha = v[0];
      dp[j] = M[o * ldm + o];
      double beta = alpha;
      if (xn2 == 0.0) {
        s_tau = 0.0;
        s_scale = 0.0;
      } else {
        beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
        s_tau = (beta - alpha) / beta;
        s_scale = 1.0 / (alpha - beta);
      }
      ep[j] = beta;
      tp[j] = s_tau;
    }
    __syncthreads();
    const double t = s_tau;
    const double sc = s_scale;
    for (int i = tid; i < m; i += blockDim.x) {
      if (t == 0.0 && i > 0) continue;
      const double vi = (i == 0) ? 1.0 : v[i] * sc;
      v[i] = vi;
      Ap[j * lda + (j + 1 + i)] = vi;  // reflector for the back-transformation
    }
    __syncthreads();
    if (t == 0.0) continue;
    // p = tau A22 v. A22 is symmetric, so p_i is column i of A22 (contiguous in
    // column-major storage) dotted with v: one warp per column, lanes along it.
    const int warp = tid >> 5, lane = tid & 31, nwarps = blockDim.x >> 5;
    for (int i = warp; i < m; i += nwarps) {
      const double* col = M + (o + 1 + i) * ldm + (o + 1);
      double acc = 0.0;
      for (int l = lane; l < m; l += 32) acc = fma(col[l], v[l], acc);
      for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
      if (lane == 0) w[i] = t * acc;
    }
    __syncthreads();
    part = 0.0;
    for (int i = tid; i < m; i += blockDim.x) part += w[i] * v[i];
    const double K = 0.5 * t * block_sum(part, red);
    for (int i = tid; i < m; i += blockDim.x) w[i] = w[i] - K * v[i];
    __syncthreads();
    // A22 -= v w^T + w v^T: one warp per column, lanes along it.
    for (int l = warp; l < m; l += nwarps) {
      double* col = M + (o + 1 + l) * ldm + (o + 1);
      const double vl = v[l], wl = w[l];
      for (int i = lane; i < m; i += 32) col[i] -= v[i] * wl + w[i] * vl;
    }
    __syncthreads();
  }
  if (tid == 0) {
    if (k >= 2) {
      const int64_t o = (k - 2) - moff;
      dp[k - 2] = M[o * ldm + o];
      ep[k - 2] = M[o * ldm + o + 1];
      tp[k - 2] = 0.0;
      dp[k - 1] = M[(o + 1) * ldm + o + 1];
    } else if (k == 1) {
      dp[0] = M[0];
    }
  }
}

// Householder tridiagonalization on a cluster of kClu CTAs with the whole matrix in
// distributed shared memory: CTA r owns the columns g = r, r + kClu, r + 2 kClu, ...
// (full length, column-major), so the shrinking trailing matrix stays spread over the
// cluster. Step j, with the same arithmetic as sytrd_kernel:
//   1. the owner of column j forms the reflector from its (already updated) column,
//      writes it to A's lower part and to every CTA's v buffer (double-buffered by the
//      parity of j, so it may be written while the previous step's update still reads
//      the other buffer); cluster barrier;
//   2. every CTA forms p_g = tau * (A22 v)_g for its own trailing columns g (a column
//      of the symmetric A22 dotted with v) and stores p_g and its share of p.v into
//      every CTA; cluster barrier;
//   3. every CTA forms w = p - (tau/2)(p.v) v in full and updates its own columns.
// Two cluster barriers per step; tau is the same in every CTA after barrier 1, so the
// skip of a zero reflector is uniform over the cluster.
constexpr int kClu = 8;
constexpr int kCluThreads = 512;

__global__ void __cluster_dims__(kClu, 1, 1) __launch_bounds__(kCluThreads, 1)
sytrd_cluster_kernel(const int32_t* __restrict__ msz, double* __restrict__ A, int64_t lda,
                     double* __restrict__ d, double* __restrict__ e, double* __restrict__ tau,
                     int64_t vec_stride, int kmax) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ double sh[];
  const int rank = static_cast<int>(cl.block_rank());
  const int p = blockIdx.x / kClu;
  const int k = msz[p];
  const int nc_max = (kmax + kClu - 1) / kClu;
  double* S = sh;                                      // own columns, ld = kmax
  double* vb = S + static_cast<int64_t>(nc_max) * kmax;  // 2 x kmax (by step parity)
  double* pall = vb + 2 * kmax;                        // p, all of it
  double* w = pall + kmax;
  double* part = w + kmax;                             // kClu shares of p.v
  double* red = part + kClu;                           // 32 reduction slots
  double* tau_s = red + 32;                            // 2 (by step parity)
  __shared__ double s_scale;
  double* Ap = A + static_cast<int64_t>(p) * lda * lda;
  double* dp = d + p * vec_stride;
  double* ep = e + p * vec_stride;
  double* tp = tau + p * vec_stride;
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31, nwarps = blockDim.x >> 5;
  const int nc = rank < k ? (k - rank + kClu - 1) / kClu : 0;  // own columns

  for (int64_t idx = tid; idx < static_cast<int64_t>(nc) * k; idx += blockDim.x) {
    const int c = static_cast<int>(idx / k), i = static_cast<int>(idx % k);
    S[static_cast<int64_t>(c) * kmax + i] = Ap[static_cast<int64_t>(rank + c * kClu) * lda + i];
  }
  cl.sync();  // every CTA runs before any writes into its shared memory

  for (int j = 0; j + 2 < k; ++j) {
    const int m = k - j - 1;
    const int buf = j & 1;
    if (rank == j % kClu) {
      const double* col = S + static_cast<int64_t>(j / kClu) * kmax;
      double part2 = 0.0;
      for (int i = 1 + tid; i < m; i += blockDim.x) part2 += col[j + 1 + i] * col[j + 1 + i];
      const double xn2 = block_sum(part2, red);
      if (tid == 0) {
        const double alpha = col[j + 1];
        double beta = alpha, t = 0.0, sc = 0.0;
        if (xn2 != 0.0) {
          beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
          t = (beta - alpha) / beta;
          sc = 1.0 / (alpha - beta);
        }
        dp[j] = col[j];
        ep[j] = beta;
        tp[j] = t;
        s_scale = sc;
        for (int q = 0; q < kClu; ++q) *cl.map_shared_rank(tau_s + buf, q) = t;
      }
      __syncthreads();
      const double sc = s_scale;
      double* vdst = vb + buf * kmax;
      for (int idx = tid; idx < m * kClu; idx += blockDim.x) {
        const int i = idx % m, q = idx / m;
        const double vi = (i == 0) ? 1.0 : col[j + 1 + i] * sc;
        *cl.map_shared_rank(vdst + i, q) = vi;
        if (q == 0) Ap[static_cast<int64_t>(j) * lda + (j + 1 + i)] = vi;
      }
    }
    cl.sync();  // barrier 1: v and tau everywhere
    const double t = tau_s[buf];
    if (t == 0.0) continue;
    const double* v = vb + buf * kmax;
    // own trailing columns: g = rank + c kClu > j
    const int c_lo = (j + 1 - rank + kClu - 1) / kClu > 0 ? (j + 1 - rank + kClu - 1) / kClu : 0;
    double share = 0.0;
    for (int c = c_lo + warp; c < nc; c += nwarps) {
      const int g = rank + c * kClu;
      const double* col = S + static_cast<int64_t>(c) * kmax + (j + 1);
      double acc = 0.0;
      for (int l = lane; l < m; l += 32) acc = fma(col[l], v[l], acc);
      for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
      const double pg = t * acc;
      if (lane < kClu) *cl.map_shared_rank(pall + (g - j - 1), lane) = pg;
      share += pg * v[g - j - 1];  // the same in every lane
    }
    if (lane == 0) red[warp] = share;
    __syncthreads();
    if (tid < kClu) {
      double s = 0.0;
      for (int i = 0; i < nwarps; ++i) s += red[i];
      *cl.map_shared_rank(part + rank, tid) = s;
    }
    cl.sync();  // barrier 2: p and the shares of p.v everywhere
    double pv = 0.0;
    for (int q = 0; q < kClu; ++q) pv += part[q];
    const double K = 0.5 * t * pv;
    for (int i = tid; i < m; i += blockDim.x) w[i] = pall[i] - K * v[i];
    __syncthreads();
    for (int c = c_lo + warp; c < nc; c += nwarps) {
      const int g = rank + c * kClu;
      double* col = S + static_cast<int64_t>(c) * kmax + (j + 1);
      const double vl = v[g - j - 1], wl = w[g - j - 1];
      for (int l = lane; l < m; l += 32) col[l] -= v[l] * wl + w[l] * vl;
    }
    __syncthreads();  // the owner of column j + 1 reads it next
  }
  if (tid == 0) {
    if (k >= 2) {
      if (rank == (k - 2) % kClu) {
        const double* col = S + static_cast<int64_t>((k - 2) / kClu) * kmax;
        dp[k - 2] = col[k - 2];
        ep[k - 2] = col[k - 1];
        tp[k - 2] = 0.0;
      }
      if (rank == (k - 1) % kClu) dp[k - 1] = S[static_cast<int64_t>((k - 1) / kClu) * kmax + k - 1];
    } else if (rank == 0) {
      dp[0] = S[0];
    }
  }
  cl.sync();  // no CTA leaves while another may still address its shared memory
}

size_t sytrd_cluster_smem(int kmax) {
  const int64_t nc_max = (kmax + kClu - 1) / kClu;
  return static_cast<size_t>((nc_max * kmax + 4 * static_cast<int64_t>(kmax) + kClu + 32 + 2) * 8);
}

__device__ __forceinline__ void gershgorin(const double* d, const double* e, int k, double& gl,
                                           double& gu, double& tnorm, double& pivmin) {
  gl = 1e308;
  gu = -1e308;
  double emax = 0.0;
  bool finite = true;
  for (int i = 0; i < k; ++i) {
    finite = finite && isfinite(d[i]) && (i + 1 >= k || isfinite(e[i]));
    const double r = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i + 1 < k ? fabs(e[i]) : 0.0);
    gl = fmin(gl, d[i] - r);
    gu = fmax(gu, d[i] + r);
    if (i + 1 < k) emax = fmax(emax, e[i] * e[i]);
  }
  if (!finite) {  // fmin/fmax drop NaN: report non-finite data through the bounds
    gl = gu = nan("");
  }
  tnorm = fmax(fabs(gl), fabs(gu));
  pivmin = kTiny * fmax(1.0, emax);
  const double pad = 2.0 * kEps * tnorm * k + 2.0 * pivmin;
  gl -= pad;
  gu += pad;
}

__device__ __forceinline__ int sturm_count(const double* d, const double* e, int k, double x,
                                           double pivmin) {
  int cnt = 0;
  double q = d[0] - x;
  if (fabs(q) < pivmin) q = -pivmin;
  cnt += q < 0.0;
  for (int i = 1; i < k; ++i) {
    q = d[i] - x - e[i - 1] * e[i - 1] / q;
    if (fabs(q) < pivmin) q = -pivmin;
    cnt += q < 0.0;
  }
  return cnt;
}

// Eigenvalue i of tridiagonal p by multisection, one CTA of kStebzThreads threads per
// eigenvalue: each round every thread takes the Sturm count at one of kStebzThreads
// interior points of [lo, hi], and the interval shrinks to the sub-interval where the
// count first passes i (7 bits per round for 128 threads, where bisection gains 1).
// One count per thread keeps each thread's chain of dependent divisions short and
// spreads the chains over every SM. info[p] = 1 for non-finite data.
constexpr int kStebzThreads = 128;

__global__ void __launch_bounds__(kStebzThreads)
stebz_kernel(const int32_t* __restrict__ msz, const double* __restrict__ d,
             const double* __restrict__ e, int64_t vec_stride, double* __restrict__ W,
             int64_t ldw, double* __restrict__ tnorm_out, int32_t* __restrict__ info) {
  __shared__ int s_first[kStebzThreads / 32];
  const int p = blockIdx.y;
  const int k = msz[p];
  const int i = blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (i >= k) return;  // the whole CTA
  const double* dp = d + p * vec_stride;
  const double* ep = e + p * vec_stride;
  double gl, gu, tnorm, pivmin;
  gershgorin(dp, ep, k, gl, gu, tnorm, pivmin);
  if (!isfinite(gl) || !isfinite(gu)) {
    if (tid == 0) {
      if (i == 0) {
        info[p] = 1;
        tnorm_out[p] = 1.0;
      }
      W[p * ldw + i] = nan("");
    }
    return;
  }
  if (i == 0 && tid == 0) tnorm_out[p] = tnorm;
  constexpr double kDen = static_cast<double>(kStebzThreads + 1);
  double lo = gl, hi = gu;
  for (int round = 0; round < 64; ++round) {
    // the same lo, hi in every thread: the loop exits uniformly
    if (hi - lo <= 2.0 * kEps * fmax(fabs(lo), fabs(hi)) + pivmin) break;
    const double x = lo + (hi - lo) * (static_cast<double>(tid + 1) / kDen);
    const bool above = sturm_count(dp, ep, k, x, pivmin) > i;
    const unsigned mask = __ballot_sync(0xffffffffu, above);
    if (lane == 0) s_first[warp] = mask ? warp * 32 + __ffs(mask) - 1 : kStebzThreads;
    __syncthreads();
    int first = kStebzThreads;  // first point with count > i
#pragma unroll
    for (int w = 0; w < kStebzThreads / 32; ++w) first = min(first, s_first[w]);
    __syncthreads();  // s_first is rewritten next round
    const double nlo =
        first == 0 ? lo : lo + (hi - lo) * (static_cast<double>(first) / kDen);
    const double nhi =
        first == kStebzThreads ? hi : lo + (hi - lo) * (static_cast<double>(first + 1) / kDen);
    if (nlo == lo && nhi == hi) break;  // no representable progress
    lo = nlo;
    hi = nhi;
  }
  if (tid == 0) W[p * ldw + i] = 0.5 * (lo + hi);
}

__device__ __forceinline__ double hash_uniform(uint64_t a, uint64_t b) {
  uint64_t z = a * 0x9E3779B97F4A7C15ull + b + 0x632BE59BD9B4E019ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return static_cast<double>(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

// LU of T - lambda I with partial pivoting (one thread). U: reciprocal diagonal u0
// (pivots smaller than `tiny` replaced by +-tiny first), first and second
// superdiagonals u1, u2 (zero past the end); L multipliers l; piv[i] = 1 where rows
// i, i+1 were swapped.
__device__ void tri_factor(const double* d, const double* e, int k, double lam, double tiny,
                           double* u0, double* u1, double* u2, double* l, double* piv) {
  auto inv_pivot = [tiny](double pv) {
    if (fabs(pv) < tiny) pv = (pv != 0.0) ? copysign(tiny, pv) : tiny;
    return 1.0 / pv;
  };
  double cur_d = d[0] - lam;
  double cur_u = k > 1 ? e[0] : 0.0;
  for (int i = 0; i + 1 < k; ++i) {
    const double sub = e[i];
    const double nd = d[i + 1] - lam;
    const double nu = (i + 2 < k) ? e[i + 1] : 0.0;
    if (fabs(cur_d) >= fabs(sub)) {
      piv[i] = 0.0;
      if (cur_d == 0.0) cur_d = tiny;
      const double mlt = sub / cur_d;
      l[i] = mlt;
      u0[i] = inv_pivot(cur_d);
      u1[i] = cur_u;
      u2[i] = 0.0;
      cur_d = nd - mlt * cur_u;
      cur_u = nu;
    } else {
      piv[i] = 1.0;
      const double mlt = cur_d / sub;
      l[i] = mlt;
      u0[i] = inv_pivot(sub);
      u1[i] = nd;
      u2[i] = nu;
      cur_d = cur_u - mlt * nd;
      cur_u = -mlt * nu;
    }
  }
  u0[k - 1] = inv_pivot(cur_d);
  u1[k - 1] = 0.0;
  u2[k - 1] = 0.0;
  if (k >= 2) u2[k - 2] = 0.0;
}

// x <- (T - lambda I)^{-1} x with the factors above (one thread). The running values
// stay in registers, so each step's chain is a few FMAs and no load waits on a store.
__device__ void tri_solve(int k, const double* u0, const double* u1, const double* u2,
                          const double* l, const double* piv, double* x) {
  double xi = x[0];
  for (int i = 0; i + 1 < k; ++i) {
    const double xn = x[i + 1];
    const double li = l[i];
    if (piv[i] != 0.0) {
      x[i] = xn;
      xi = xi - li * xn;
    } else {
      x[i] = xi;
      xi = xn - li * xi;
    }
  }
  x[k - 1] = xi;
  double x1 = 0.0, x2 = 0.0;  // x[i + 1], x[i + 2]
  for (int i = k - 1; i >= 0; --i) {
    const double s = x[i] - u1[i] * x1 - u2[i] * x2;
    const double r = s * u0[i];
    x[i] = r;
    x2 = x1;
    x1 = r;
  }
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// One warp per cluster start: eigenvectors of tridiagonal p into Z_T (column-major,
// ldz) for the cluster's eigenvalues. Scratch: 6 k doubles per eigenvalue index.
__global__ void stein_kernel(const int32_t* __restrict__ msz, const double* __restrict__ d,
                             const double* __restrict__ e, int64_t vec_stride,
                             const double* __restrict__ W, int64_t ldw,
                             const double* __restrict__ tnorm_in, double* __restrict__ Z,
                             int64_t ldz, double* __restrict__ scratch, int64_t scratch_stride) {
  const int p = blockIdx.y;
  const int k = msz[p];
  const int t0 = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (t0 >= k) return;
  double* Zp = Z + static_cast<int64_t>(p) * ldz * ldz;
  if (k == 1) {
    if (lane == 0) Zp[0] = 1.0;
    return;
  }
  const double* dp = d + p * vec_stride;
  const double* ep = e + p * vec_stride;
  const double* wp = W + p * ldw;
  const double tnorm = tnorm_in[p];
  const double gap = kClusterTol * tnorm;
  if (t0 > 0 && wp[t0] - wp[t0 - 1] <= gap) return;  // not the first of its cluster
  int t1 = t0;
  while (t1 + 1 < k && wp[t1 + 1] - wp[t1] <= gap) ++t1;
  double* s = scratch + (static_cast<int64_t>(p) * ldz + t0) * scratch_stride;
  double *u0 = s, *u1 = s + k, *u2 = s + 2 * k, *l = s + 3 * k, *piv = s + 4 * k, *x = s + 5 * k;
  const double tiny = kEps * fmax(tnorm, kTiny);
  for (int t = t0; t <= t1; ++t) {
    if (lane == 0) tri_factor(dp, ep, k, wp[t], tiny, u0, u1, u2, l, piv);
    for (int i = lane; i < k; i += 32) x[i] = hash_uniform(static_cast<uint64_t>(t) + 1, i);
    __syncwarp();
    for (int it = 0; it < 3; ++it) {
      // scale to max |x| = 1, solve, orthogonalize against the cluster's earlier
      // vectors, normalize
      double mx = 0.0;
      for (int i = lane; i < k; i += 32) mx = fmax(mx, fabs(x[i]));
      for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      const double inv = mx > 0.0 ? 1.0 / mx : 1.0;
      for (int i = lane; i < k; i += 32) x[i] *= inv;
      __syncwarp();
      if (lane == 0) tri_solve(k, u0, u1, u2, l, piv, x);
      __syncwarp();
      for (int q = t0; q < t; ++q) {
        const double* zq = Zp + static_cast<int64_t>(q) * ldz;
        double dot = 0.0;
        for (int i = lane; i < k; i += 32) dot += zq[i] * x[i];
        dot = warp_sum(dot);
        for (int i = lane; i < k; i += 32) x[i] -= dot * zq[i];
        __syncwarp();
      }
      double nn = 0.0;
      for (int i = lane; i < k; i += 32) nn += x[i] * x[i];
      nn = warp_sum(nn);
      const double sc = nn > 0.0 ? 1.0 / sqrt(nn) : 0.0;
      for (int i = lane; i < k; i += 32) x[i] *= sc;
      __syncwarp();
    }
    double* zt = Zp + static_cast<int64_t>(t) * ldz;
    for (int i = lane; i < k; i += 32) zt[i] = x[i];
    __syncwarp();
  }
}

// Z <- H_0 ... H_{k-3} Z (reflectors in A's strictly lower part, v0 = 1 stored),
// one warp per column of Z.
__global__ void ormtr_kernel(const int32_t* __restrict__ msz, const double* __restrict__ A,
                             int64_t lda, const double* __restrict__ tau, int64_t vec_stride,
                             double* __restrict__ Z, int64_t ldz) {
  const int p = blockIdx.y;
  const int k = msz[p];
  const int c = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (c >= k) return;
  const double* Ap = A + static_cast<int64_t>(p) * lda * lda;
  const double* tp = tau + p * vec_stride;
  double* z = Z + static_cast<int64_t>(p) * ldz * ldz + static_cast<int64_t>(c) * ldz;
  for (int j = k - 3; j >= 0; --j) {
    const double t = tp[j];
    if (t == 0.0) continue;
    const double* v = Ap + static_cast<int64_t>(j) * lda + (j + 1);
    double s = 0.0;
    for (int i = lane; i < k - j - 1; i += 32) s += v[i] * z[j + 1 + i];
    s = warp_sum(s) * t;
    for (int i = lane; i < k - j - 1; i += 32) z[j + 1 + i] -= s * v[i];
    __syncwarp();
  }
}

// As ormtr_kernel with the columns held in shared memory: a CTA takes kOrmCols columns
// of Z (a warp each) and streams the reflectors through shared memory kOrmChunk at a
// time, so each reflector is read from global memory once per CTA and every dot
// product and update runs on shared memory.
constexpr int kOrmCols = 8;
constexpr int kOrmChunk = 8;

__global__ void __launch_bounds__(kOrmCols * 32)
ormtr_smem_kernel(const int32_t* __restrict__ msz, const double* __restrict__ A, int64_t lda,
                  const double* __restrict__ tau, int64_t vec_stride, double* __restrict__ Z,
                  int64_t ldz, int kmax) {
  extern __shared__ double sh[];
  const int p = blockIdx.y;
  const int k = msz[p];
  const int c0 = blockIdx.x * kOrmCols;
  if (c0 >= k) return;  // the whole CTA
  double* zc = sh;                                           // kOrmCols x kmax
  double* vr = zc + static_cast<int64_t>(kOrmCols) * kmax;   // kOrmChunk x kmax
  double* tr = vr + static_cast<int64_t>(kOrmChunk) * kmax;  // kOrmChunk
  const double* Ap = A + static_cast<int64_t>(p) * lda * lda;
  const double* tp = tau + p * vec_stride;
  double* Zp = Z + static_cast<int64_t>(p) * ldz * ldz;
  const int ncols = min(kOrmCols, k - c0);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int idx = tid; idx < ncols * k; idx += blockDim.x) {
    const int c = idx / k, i = idx % k;
    zc[static_cast<int64_t>(c) * kmax + i] = Zp[static_cast<int64_t>(c0 + c) * ldz + i];
  }
  for (int jhi = k - 3; jhi >= 0; jhi -= kOrmChunk) {
    const int jlo = max(0, jhi - kOrmChunk + 1);
    __syncthreads();  // the previous chunk is applied
    for (int j = jhi - (tid / 32); j >= jlo; j -= blockDim.x / 32) {
      const int m = k - j - 1;
      double* dst = vr + static_cast<int64_t>(jhi - j) * kmax;
      const double* src = Ap + static_cast<int64_t>(j) * lda + (j + 1);
      for (int i = lane; i < m; i += 32) dst[i] = src[i];
      if (lane == 0) tr[jhi - j] = tp[j];
    }
    __syncthreads();
    if (warp < ncols) {
      double* z = zc + static_cast<int64_t>(warp) * kmax;
      for (int j = jhi; j >= jlo; --j) {
        const double t = tr[jhi - j];
        if (t == 0.0) continue;
        const double* v = vr + static_cast<int64_t>(jhi - j) * kmax;
        const int m = k - j - 1;
        double s = 0.0;
        for (int i = lane; i < m; i += 32) s = fma(v[i], z[j + 1 + i], s);
        s = warp_sum(s) * t;
        for (int i = lane; i < m; i += 32) z[j + 1 + i] -= s * v[i];
        __syncwarp();
      }
    }
  }
  __syncthreads();
  for (int idx = tid; idx < ncols * k; idx += blockDim.x) {
    const int c = idx / k, i = idx % k;
    Zp[static_cast<int64_t>(c0 + c) * ldz + i] = zc[static_cast<int64_t>(c) * kmax + i];
  }
}

size_t ormtr_smem_bytes(int kmax) {
  return static_cast<size_t>((static_cast<int64_t>(kOrmCols + kOrmChunk) * kmax + kOrmChunk) * 8);
}

struct SyevdWs {
  double *d, *e, *tau, *tnorm, *scratch;
  int32_t* msz;
  size_t total;
  int64_t vec_stride, scratch_stride;
  SyevdWs(void* base, int count, int64_t lda) {
    vec_stride = lda;
    scratch_stride = 6 * lda;
    char* p = static_cast<char*>(base);
    size_t off = 0;
    auto take = [&](size_t b) {
      char* q = p ? p + off : nullptr;
      off += (b + 255) / 256 * 256;
      return q;
    };
    d = reinterpret_cast<double*>(take(sizeof(double) * count * lda));
    e = reinterpret_cast<double*>(take(sizeof(double) * count * lda));
    tau = reinterpret_cast<double*>(take(sizeof(double) * count * lda));
    tnorm = reinterpret_cast<double*>(take(sizeof(double) * count));
    msz = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * count));
    scratch = reinterpret_cast<double*>(take(sizeof(double) * count * lda * scratch_stride));
    total = off;
  }
};

int smem_optin() {
  int dev = 0, optin = 0;
  FE_CHECK_CUDA(cudaGetDevice(&dev));
  FE_CHECK_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  return optin;
}

int current_device() {
  int dev = 0;
  FE_CHECK_CUDA(cudaGetDevice(&dev));
  return dev;
}

// cudaFuncSetAttribute(MaxDynamicSharedMemorySize) once per (kernel slot, device).
void set_max_smem_once(const void* kernel, int bytes, int dev, int slot) {
  static std::mutex mu;
  static bool done[4][64] = {};
  std::lock_guard<std::mutex> lock(mu);
  const bool tracked = dev >= 0 && dev < 64;
  if (tracked && done[slot][dev]) return;
  FE_CHECK_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  if (tracked) done[slot][dev] = true;
}

// Tridiagonalization kernel: 0 = by size (below), 1 = one CTA per matrix, 2 = the
// 8-CTA cluster wherever it fits.
int g_sytrd_mode = 0;
constexpr int kClusterMinDim = 0;

// The cluster tridiagonalization runs when its shared memory fits and the device can
// co-schedule one cluster of kClu such CTAs (asked once per device and size).
bool use_cluster_sytrd(int kmax, int optin, int dev) {
  if (g_sytrd_mode == 1) return false;
  if (g_sytrd_mode == 0 && kmax < kClusterMinDim) return false;
  const size_t smem = sytrd_cluster_smem(kmax);
  if (smem + 1024 > static_cast<size_t>(optin)) return false;
  set_max_smem_once(reinterpret_cast<const void*>(sytrd_cluster_kernel), optin - 256, dev, 1);
  static std::mutex mu;
  static std::map<std::pair<int, size_t>, bool> known;
  std::lock_guard<std::mutex> lock(mu);
  const auto key = std::make_pair(dev, smem);
  auto it = known.find(key);
  if (it != known.end()) return it->second;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(kClu, 1, 1);
  cfg.blockDim = dim3(kCluThreads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  int clusters = 0;
  const cudaError_t err =
      cudaOccupancyMaxActiveClusters(&clusters, sytrd_cluster_kernel, &cfg);
  if (err != cudaSuccess) (void)cudaGetLastError();
  const bool ok = err == cudaSuccess && clusters >= 1;
  known[key] = ok;
  return ok;
}

}  // namespace

namespace {
void syevd_batched_prepared(int count, int kmax, const SyevdWs& w, double* A, int64_t lda,
                            double* W, double* Z, int32_t* info, cudaStream_t s);
__global__ void fill_sizes_kernel(int32_t* msz, int count, int32_t k) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) msz[i] = k;
}
}  // namespace

size_t syevd_workspace_bytes(int count, int64_t lda) {
  return SyevdWs(nullptr, count, lda).total;
}

void syevd_batched(int count, const int32_t* m_host, double* A, int64_t lda, double* W,
                   double* Z, int32_t* info, void* ws, size_t ws_bytes, cudaStream_t s) {
  FE_REQUIRE(count >= 1, "syevd: count must be >= 1");
  int kmax = 0;
  for (int p = 0; p < count; ++p) {
    FE_REQUIRE(m_host[p] >= 1 && m_host[p] <= lda, "syevd: sizes must be in [1, lda]");
    kmax = std::max(kmax, m_host[p]);
  }
  FE_REQUIRE(kmax <= 8192, "syevd: matrices larger than 8192 are not supported");
  SyevdWs w(ws, count, lda);
  FE_REQUIRE(ws && ws_bytes >= w.total, "syevd: workspace too small");
  FE_CHECK_CUDA(cudaMemcpyAsync(w.msz, m_host, sizeof(int32_t) * count, cudaMemcpyHostToDevice, s));
  syevd_batched_prepared(count, kmax, w, A, lda, W, Z, info, s);
}

// All `count` matrices of size k: the sizes are written on the device, so the whole
// sequence is stream-capturable (grouped solves replay it from a CUDA graph).
void syevd_batched_uniform(int count, int64_t k, double* A, int64_t lda, double* W, double* Z,
                           int32_t* info, void* ws, size_t ws_bytes, cudaStream_t s) {
  FE_REQUIRE(count >= 1 && k >= 1 && k <= lda && k <= 8192, "syevd: invalid batch shape");
  SyevdWs w(ws, count, lda);
  FE_REQUIRE(ws && ws_bytes >= w.total, "syevd: workspace too small");
  fill_sizes_kernel<<<(count + 127) / 128, 128, 0, s>>>(w.msz, count, static_cast<int32_t>(k));
  check_launch("fill_sizes_kernel");
  syevd_batched_prepared(count, static_cast<int>(k), w, A, lda, W, Z, info, s);
}

namespace {
void syevd_batched_prepared(int count, int kmax, const SyevdWs& w, double* A, int64_t lda,
                            double* W, double* Z, int32_t* info, cudaStream_t s) {
  FE_CHECK_CUDA(cudaMemsetAsync(info, 0, sizeof(int32_t) * count, s));
  const int optin = smem_optin();
  const int dev = current_device();
  if (use_cluster_sytrd(kmax, optin, dev)) {
    sytrd_cluster_kernel<<<count * kClu, kCluThreads, sytrd_cluster_smem(kmax), s>>>(
        w.msz, A, lda, w.d, w.e, w.tau, w.vec_stride, kmax);
    check_launch("sytrd_cluster_kernel");
  } else {
    // dynamic shared memory: 2 vectors + reduction slots + the trailing-matrix tile
    const int64_t fixed = (2 * static_cast<int64_t>(kmax) + 32) * 8;
    const int64_t tile_cap = std::max<int64_t>(0, (optin - fixed - 1024) / 8);
    const size_t smem = static_cast<size_t>(fixed + tile_cap * 8);
    set_max_smem_once(reinterpret_cast<const void*>(sytrd_kernel), optin - 256, dev, 0);
    sytrd_kernel<<<count, kTrdThreads, smem, s>>>(w.msz, A, lda, w.d, w.e, w.tau, w.vec_stride,
                                                  kmax, tile_cap);
    check_launch("sytrd_kernel");
  }
  stebz_kernel<<<dim3(kmax, count), kStebzThreads, 0, s>>>(w.msz, w.d, w.e, w.vec_stride, W,
                                                            lda, w.tnorm, info);
  check_launch("stebz_kernel");
  FE_CHECK_CUDA(cudaMemsetAsync(Z, 0, sizeof(double) * count * lda * lda, s));
  stein_kernel<<<dim3((kmax + 3) / 4, count), 128, 0, s>>>(w.msz, w.d, w.e, w.vec_stride, W, lda,
                                                           w.tnorm, Z, lda, w.scratch,
                                                           w.scratch_stride);
  check_launch("stein_kernel");
  const size_t orm_smem = ormtr_smem_bytes(kmax);
  if (orm_smem + 1024 <= static_cast<size_t>(optin)) {
    set_max_smem_once(reinterpret_cast<const void*>(ormtr_smem_kernel), optin - 256, dev, 2);
    ormtr_smem_kernel<<<dim3((kmax + kOrmCols - 1) / kOrmCols, count), kOrmCols * 32, orm_smem,
                        s>>>(w.msz, A, lda, w.tau, w.vec_stride, Z, lda, kmax);
    check_launch("ormtr_smem_kernel");
  } else {
    ormtr_kernel<<<dim3((kmax + 7) / 8, count), 256, 0, s>>>(w.msz, A, lda, w.tau, w.vec_stride,
                                                             Z, lda);
    check_launch("ormtr_kernel");
  }
}
}  // namespace

size_t syevd_single_workspace_bytes(int64_t k) {
  // reflector copy of A and the eigenvectors (k x k each), vectors, scratch
  const size_t mat = (static_cast<size_t>(k) * k * sizeof(double) + 255) / 256 * 256;
  return 2 * mat + syevd_workspace_bytes(1, k);
}

void syevd_single(double* A, int64_t lda, int64_t k, double* W, int32_t* info, void* ws,
                  size_t ws_bytes, cudaStream_t s) {
  FE_REQUIRE(A && W && info, "null argument");
  FE_REQUIRE(k >= 1 && lda >= k, "syevd: need 1 <= k <= lda");
  const size_t need = syevd_single_workspace_bytes(k);
  FE_REQUIRE(ws && ws_bytes >= need,
             "syevd: workspace too small (need " + std::to_string(need) + " bytes)");
  const size_t mat = (static_cast<size_t>(k) * k * sizeof(double) + 255) / 256 * 256;
  double* Ak = static_cast<double*>(ws);
  double* Zk = reinterpret_cast<double*>(static_cast<char*>(ws) + mat);
  char* rest = static_cast<char*>(ws) + 2 * mat;
  FE_CHECK_CUDA(cudaMemcpy2DAsync(Ak, k * sizeof(double), A, lda * sizeof(double),
                                  k * sizeof(double), k, cudaMemcpyDeviceToDevice, s));
  const int32_t m = static_cast<int32_t>(k);
  syevd_batched(1, &m, Ak, k, W, Zk, info, rest, ws_bytes - 2 * mat, s);
  FE_CHECK_CUDA(cudaMemcpy2DAsync(A, lda * sizeof(double), Zk, k * sizeof(double),
                                  k * sizeof(double), k, cudaMemcpyDeviceToDevice, s));
}

}  // namespace fe

extern "C" int fe_set_syevd_kernel(int32_t mode) {
  return fe::guarded("fe_set_syevd_kernel", [&] {
    FE_REQUIRE(mode >= 0 && mode <= 2, "syevd kernel mode must be 0, 1 or 2");
    fe::g_sytrd_mode = mode;
  });
}

extern "C" size_t fe_syevd_f64_workspace_bytes(int64_t k) {
  return k <= 0 ? 0 : fe::syevd_single_workspace_bytes(k);
}

extern "C" int fe_syevd_f64(double* A, int64_t lda, int64_t k, double* W, int32_t* info,
                            void* workspace, size_t workspace_bytes, void* stream) {
  return fe::guarded("fe_syevd_f64", [&] {
    fe::syevd_single(A, lda, k, W, info, workspace, workspace_bytes, fe::as_stream(stream));
  });
}
