// Symmetric eigensolver for small dense FP64 matrices on the device (the projected
// k-by-k problems of Rayleigh-Ritz and Krylov-Schur). It replaces the Dsyevd call
// of the reference's GPU path (src/gpu/CudaLanczosWorkspace.cpp:155-157) and the
// host Eigen SelfAdjointEigenSolver of its CPU path (src/core/RitzExtraction.cpp:104).
//
// Four kernels, each batched over matrices (matrix p: A + p*lda*lda, size m[p]):
//   1. sytrd: Householder tridiagonalization, one CTA per matrix. Step j reflects
//      column j below the diagonal (dlarfg convention: beta = -sign(alpha)||x||,
//      tau = (beta - alpha)/beta, v = x/(alpha - beta), v0 = 1), then
//      p = tau A22 v, w = p - (tau/2)(p.v) v, A22 -= v w^T + w v^T (both triangles
//      kept). The trailing matrix moves into shared memory once it fits. The
//      reflectors stay in A's strictly lower part for step 4.
//   2. stebz: every eigenvalue of the tridiagonal by multisection on its Sturm
//      count, one warp per eigenvalue index (ascending order by construction).
//   3. stein: eigenvectors of the tridiagonal by inverse iteration (LU of T - lambda
//      I with partial pivoting, tiny pivots replaced by eps*||T||, three solves from
//      a hashed start vector), one warp per cluster of eigenvalues closer than
//      1e-4 ||T||; members of a cluster are orthogonalized against the earlier ones
//      (modified Gram-Schmidt) after every solve.
//   4. ormtr: Z = H_0 H_1 ... H_{m-3} Z_T, one warp per column of Z.
#include <algorithm>
#include <cmath>
#include <string>

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

// Eigenvalue i of tridiagonal p by multisection, one warp per eigenvalue: each round
// the 32 lanes take Sturm counts at 32 interior points of [lo, hi] and the interval
// shrinks to the sub-interval where the count passes i (5 bits per round instead of
// bisection's 1). info[p] = 1 for non-finite data.
__global__ void stebz_kernel(const int32_t* __restrict__ msz, const double* __restrict__ d,
                             const double* __restrict__ e, int64_t vec_stride,
                             double* __restrict__ W, int64_t ldw, double* __restrict__ tnorm_out,
                             int32_t* __restrict__ info) {
  const int p = blockIdx.y;
  const int k = msz[p];
  const int i = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (i >= k) return;
  const double* dp = d + p * vec_stride;
  const double* ep = e + p * vec_stride;
  double gl, gu, tnorm, pivmin;
  gershgorin(dp, ep, k, gl, gu, tnorm, pivmin);
  if (!isfinite(gl) || !isfinite(gu)) {
    if (i == 0 && lane == 0) {
      info[p] = 1;
      tnorm_out[p] = 1.0;
    }
    if (lane == 0) W[p * ldw + i] = nan("");
    return;
  }
  if (i == 0 && lane == 0) tnorm_out[p] = tnorm;
  double lo = gl, hi = gu;
  for (int round = 0; round < 64; ++round) {
    if (hi - lo <= 2.0 * kEps * fmax(fabs(lo), fabs(hi)) + pivmin) break;
    const double x = lo + (hi - lo) * (static_cast<double>(lane + 1) / 33.0);
    const bool above = sturm_count(dp, ep, k, x, pivmin) > i;
    const unsigned mask = __ballot_sync(0xffffffffu, above);
    const int first = mask ? __ffs(mask) - 1 : 32;
    const double x_first = __shfl_sync(0xffffffffu, x, first < 32 ? first : 31);
    const double x_prev = __shfl_sync(0xffffffffu, x, first > 0 ? first - 1 : 0);
    const double nlo = first == 0 ? lo : x_prev;
    const double nhi = first < 32 ? x_first : hi;
    if (nlo == lo && nhi == hi) break;  // no representable progress
    lo = nlo;
    hi = nhi;
  }
  if (lane == 0) W[p * ldw + i] = 0.5 * (lo + hi);
}

__device__ __forceinline__ double hash_uniform(uint64_t a, uint64_t b) {
  uint64_t z = a * 0x9E3779B97F4A7C15ull + b + 0x632BE59BD9B4E019ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return static_cast<double>(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

// LU of T - lambda I with partial pivoting (one thread). U: diagonal u0, first and
// second superdiagonals u1, u2; L multipliers l; piv[i] = 1 where rows i, i+1 swapped.
__device__ void tri_factor(const double* d, const double* e, int k, double lam, double tiny,
                           double* u0, double* u1, double* u2, double* l, double* piv) {
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
      u0[i] = cur_d;
      u1[i] = cur_u;
      u2[i] = 0.0;
      cur_d = nd - mlt * cur_u;
      cur_u = nu;
    } else {
      piv[i] = 1.0;
      const double mlt = cur_d / sub;
      l[i] = mlt;
      u0[i] = sub;
      u1[i] = nd;
      u2[i] = nu;
      cur_d = cur_u - mlt * nd;
      cur_u = -mlt * nu;
    }
  }
  if (fabs(cur_d) < tiny) cur_d = (cur_d != 0.0) ? copysign(tiny, cur_d) : tiny;
  u0[k - 1] = cur_d;
}

// x <- (T - lambda I)^{-1} x with the factors above (one thread).
__device__ void tri_solve(int k, double tiny, const double* u0, const double* u1,
                          const double* u2, const double* l, const double* piv, double* x) {
  for (int i = 0; i + 1 < k; ++i) {
    if (piv[i] != 0.0) {
      const double a = x[i], b = x[i + 1];
      x[i] = b;
      x[i + 1] = a - l[i] * b;
    } else {
      x[i + 1] -= l[i] * x[i];
    }
  }
  for (int i = k - 1; i >= 0; --i) {
    double s = x[i];
    if (i + 1 < k) s -= u1[i] * x[i + 1];
    if (i + 2 < k) s -= u2[i] * x[i + 2];
    double pv = u0[i];
    if (fabs(pv) < tiny) pv = (pv != 0.0) ? copysign(tiny, pv) : tiny;
    x[i] = s / pv;
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
      if (lane == 0) tri_solve(k, tiny, u0, u1, u2, l, piv, x);
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
  FE_CHECK_CUDA(cudaMemsetAsync(info, 0, sizeof(int32_t) * count, s));
  const int optin = smem_optin();
  // dynamic shared memory: 2 vectors + reduction slots + the trailing-matrix tile
  const int64_t fixed = (2 * static_cast<int64_t>(kmax) + 32) * 8;
  const int64_t tile_cap = std::max<int64_t>(0, (optin - fixed - 1024) / 8);
  const size_t smem = static_cast<size_t>(fixed + tile_cap * 8);
  static bool attr = false;
  if (!attr) {
    FE_CHECK_CUDA(cudaFuncSetAttribute(sytrd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       optin - 256));
    attr = true;
  }
  sytrd_kernel<<<count, kTrdThreads, smem, s>>>(w.msz, A, lda, w.d, w.e, w.tau, w.vec_stride, kmax,
                                                tile_cap);
  check_launch("sytrd_kernel");
  stebz_kernel<<<dim3((kmax + 3) / 4, count), 128, 0, s>>>(w.msz, w.d, w.e, w.vec_stride, W, lda,
                                                            w.tnorm, info);
  check_launch("stebz_kernel");
  FE_CHECK_CUDA(cudaMemsetAsync(Z, 0, sizeof(double) * count * lda * lda, s));
  stein_kernel<<<dim3((kmax + 3) / 4, count), 128, 0, s>>>(w.msz, w.d, w.e, w.vec_stride, W, lda,
                                                           w.tnorm, Z, lda, w.scratch,
                                                           w.scratch_stride);
  check_launch("stein_kernel");
  ormtr_kernel<<<dim3((kmax + 7) / 8, count), 256, 0, s>>>(w.msz, A, lda, w.tau, w.vec_stride, Z,
                                                           lda);
  check_launch("ormtr_kernel");
}

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

extern "C" size_t fe_syevd_f64_workspace_bytes(int64_t k) {
  return k <= 0 ? 0 : fe::syevd_single_workspace_bytes(k);
}

extern "C" int fe_syevd_f64(double* A, int64_t lda, int64_t k, double* W, int32_t* info,
                            void* workspace, size_t workspace_bytes, void* stream) {
  return fe::guarded("fe_syevd_f64", [&] {
    fe::syevd_single(A, lda, k, W, info, workspace, workspace_bytes, fe::as_stream(stream));
  });
}
