// CSR block SpMM and the fused Chebyshev three-term step for sm_100a.
//
// Replaces CudaCsrMatrix::apply_block (src/gpu/CudaCsrMatrix.cpp:196-223), which
// runs one cuSPARSE SpMV per column and so streams the CSR arrays once per
// column, and the copy/SpMV/axpy sequence of ChebyshevSolver::chebyshev_filter
// (src/ChebyshevSolver.cpp:243-256), which makes about five passes over the
// block per filter step.
//
// Layout: the dense blocks are row-major slabs, so the b values a CSR row
// needs from one neighbour are contiguous. A group of G lanes owns one row;
// each lane owns CPL 128-bit vectors of that row's b columns. Nonzeros are
// fetched G at a time (one coalesced load of colind/values per group) and
// broadcast with warp shuffles; every neighbour row of X is then read with
// fully coalesced 128-bit loads. Accumulation is in the storage precision
// (FP32 blocks: FP32 values and accumulators; FP64 blocks: FP64). The epilogue
// fuses y = alpha*acc + gamma*x_row + beta*z_row and writes y once, which is
// the whole Chebyshev step.
//
// Algorithmic bytes per launch (the roofline figure): nnz*(s+4) + 4*(n+1) +
// 2*n*b*s for SpMM (X read once, Y written once), plus n*b*s for each of the
// gamma (X row re-read, an L2 hit) and beta (Z read) terms that are active.

#include "fe_common.cuh"

#include <cmath>
#include <mutex>

#include <algorithm>

namespace fe {
namespace {

template <typename T>
struct VecT;
template <>
struct VecT<float> {
  using type = float4;
  static constexpr int width = 4;
};
template <>
struct VecT<double> {
  using type = double2;
  static constexpr int width = 2;
};

template <typename T, int VEC>
struct Pack {
  T v[VEC];
};

// Vector types by total width: 16 bytes (float4 / double2), 8 bytes (float2 /
// double), 4 bytes (float).
template <typename T, int VEC>
struct Raw;
template <> struct Raw<float, 4> { using type = float4; };
template <> struct Raw<float, 2> { using type = float2; };
template <> struct Raw<float, 1> { using type = float; };
template <> struct Raw<double, 2> { using type = double2; };
template <> struct Raw<double, 1> { using type = double; };

template <typename T, int VEC>
__device__ __forceinline__ Pack<T, VEC> unpack(const typename Raw<T, VEC>::type& t) {
  Pack<T, VEC> r;
  if constexpr (VEC == 4) {
    r.v[0] = t.x; r.v[1] = t.y; r.v[2] = t.z; r.v[3] = t.w;
  } else if constexpr (VEC == 2) {
    r.v[0] = t.x; r.v[1] = t.y;
  } else {
    r.v[0] = t;
  }
  return r;
}

template <typename T, int VEC>
__device__ __forceinline__ Pack<T, VEC> load_pack(const T* p) {
  using R = typename Raw<T, VEC>::type;
  return unpack<T, VEC>(__ldg(reinterpret_cast<const R*>(p)));
}

// Load bypassing L1 (cached in L2 only), for blocks other SMs rewrite during a launch.
template <typename T, int VEC>
__device__ __forceinline__ Pack<T, VEC> load_pack_cg(const T* p) {
  using R = typename Raw<T, VEC>::type;
  return unpack<T, VEC>(__ldcg(reinterpret_cast<const R*>(p)));
}

// Plain (coherent) load for blocks that may alias the output.
template <typename T, int VEC>
__device__ __forceinline__ Pack<T, VEC> load_pack_rw(const T* p) {
  using R = typename Raw<T, VEC>::type;
  return unpack<T, VEC>(*reinterpret_cast<const R*>(p));
}

template <typename T, int VEC>
__device__ __forceinline__ void store_pack(T* p, const Pack<T, VEC>& r) {
  using R = typename Raw<T, VEC>::type;
  R t;
  if constexpr (VEC == 4) {
    t.x = r.v[0]; t.y = r.v[1]; t.z = r.v[2]; t.w = r.v[3];
  } else if constexpr (VEC == 2) {
    t.x = r.v[0]; t.y = r.v[1];
  } else {
    t = r.v[0];
  }
  *reinterpret_cast<R*>(p) = t;
}

constexpr int kThreads = 256;

// Y[row, c0:c1] = alpha * sum_k a_k X[col_k, c0:c1] + gamma * X[row, c0:c1]
//                 + beta * Z[row, c0:c1]
// blockIdx.y selects a column panel of width G*CPL*VEC.
template <typename T, int VEC, int G, int CPL>
__global__ void __launch_bounds__(kThreads)
csr_spmm_kernel(int64_t nrows, const int32_t* __restrict__ rowptr,
                const int32_t* __restrict__ colind, const T* __restrict__ vals,
                const T* __restrict__ X, int64_t ldx, T* Y, int64_t ldy, const T* Z,
                int64_t ldz, int ncols, T alpha, T gamma, T beta, int use_gamma,
                int use_beta) {
  constexpr int kRowsPerBlock = kThreads / G;
  const int group = threadIdx.x / G;
  const int lane = threadIdx.x % G;
  const int64_t row = static_cast<int64_t>(blockIdx.x) * kRowsPerBlock + group;
  if (row >= nrows) return;  // whole group leaves together
  const int panel0 = blockIdx.y * (G * CPL * VEC);
  const int nvec = (min(ncols - panel0, G * CPL * VEC) + VEC - 1) / VEC;

  unsigned mask;
  if constexpr (G == 32) {
    mask = 0xffffffffu;
  } else {
    const int warp_lane = threadIdx.x & 31;
    mask = ((1u << G) - 1u) << (warp_lane - lane);
  }

  T acc[CPL][VEC];
#pragma unroll
  for (int i = 0; i < CPL; ++i)
#pragma unroll
    for (int e = 0; e < VEC; ++e) acc[i][e] = T(0);

  const int start = __ldg(rowptr + row);
  const int end = __ldg(rowptr + row + 1);
  const T* Xp = X + panel0;
  for (int base = start; base < end; base += G) {
    const int k = base + lane;
    int c = 0;
    T a = T(0);
    if (k < end) {
      c = __ldg(colind + k);
      a = __ldg(vals + k);
    }
    const int cnt = min(G, end - base);
    int t = 0;
    // Two neighbours per trip: independent loads in flight.
    for (; t + 1 < cnt; t += 2) {
      const int c0 = __shfl_sync(mask, c, t, G);
      const T a0 = __shfl_sync(mask, a, t, G);
      const int c1 = __shfl_sync(mask, c, t + 1, G);
      const T a1 = __shfl_sync(mask, a, t + 1, G);
      const T* x0 = Xp + static_cast<int64_t>(c0) * ldx;
      const T* x1 = Xp + static_cast<int64_t>(c1) * ldx;
      Pack<T, VEC> p0[CPL], p1[CPL];
#pragma unroll
      for (int i = 0; i < CPL; ++i) {
        const int v = lane + i * G;
        if (v < nvec) {
          p0[i] = load_pack<T, VEC>(x0 + v * VEC);
          p1[i] = load_pack<T, VEC>(x1 + v * VEC);
        }
      }
#pragma unroll
      for (int i = 0; i < CPL; ++i) {
        const int v = lane + i * G;
        if (v < nvec) {
#pragma unroll
          for (int e = 0; e < VEC; ++e) {
            acc[i][e] = fma(a0, p0[i].v[e], acc[i][e]);
            acc[i][e] = fma(a1, p1[i].v[e], acc[i][e]);
          }
        }
      }
    }
    if (t < cnt) {
      const int c0 = __shfl_sync(mask, c, t, G);
      const T a0 = __shfl_sync(mask, a, t, G);
      const T* x0 = Xp + static_cast<int64_t>(c0) * ldx;
#pragma unroll
      for (int i = 0; i < CPL; ++i) {
        const int v = lane + i * G;
        if (v < nvec) {
          Pack<T, VEC> p = load_pack<T, VEC>(x0 + v * VEC);
#pragma unroll
          for (int e = 0; e < VEC; ++e) acc[i][e] = fma(a0, p.v[e], acc[i][e]);
        }
      }
    }
  }

  T* yrow = Y + row * ldy + panel0;
  const T* xrow = X + row * ldx + panel0;
  const T* zrow = use_beta ? Z + row * ldz + panel0 : nullptr;
#pragma unroll
  for (int i = 0; i < CPL; ++i) {
    const int v = lane + i * G;
    if (v < nvec) {
      Pack<T, VEC> out;
#pragma unroll
      for (int e = 0; e < VEC; ++e) out.v[e] = alpha * acc[i][e];
      if (use_gamma) {
        Pack<T, VEC> xr = load_pack<T, VEC>(xrow + v * VEC);
#pragma unroll
        for (int e = 0; e < VEC; ++e) out.v[e] = fma(gamma, xr.v[e], out.v[e]);
      }
      if (use_beta) {
        Pack<T, VEC> zr = load_pack_rw<T, VEC>(zrow + v * VEC);
#pragma unroll
        for (int e = 0; e < VEC; ++e) out.v[e] = fma(beta, zr.v[e], out.v[e]);
      }
      store_pack<T, VEC>(yrow + v * VEC, out);
    }
  }
}

// Library-default status word of the SpMM kernels' bounded waits (fe_device_status).
__device__ int g_spmm_status = 0;

// ---------------------------------------------------------------------------
// Row-batched register kernel: one warp per row for slabs of >= 32 vectors.
//
// The loop kernel above waits on a chain of dependent loads per row (rowptr ->
// colind -> two neighbours per trip -> ... -> Z). Here the whole row is issued at
// once: the neighbour rows of X (up to NZ nonzeros, all in registers) and the
// Z row are loaded together, while the CSR metadata of the next row (colind and
// values) and the row pointers of the row after it are prefetched. Each row then
// costs about one memory round trip, and a warp keeps NZ*CPL 128-bit loads per
// lane in flight. gamma is folded into the diagonal coefficient
// (alpha*a_ii + gamma); a row without a stored diagonal loads its X row.
// Columns are split into panels of at most 96 vectors (CPL <= 3).
// ---------------------------------------------------------------------------
// With CORR, every output also gains delta[j] * R[row, j] (the correction term of the
// refined filter, see csr_spmm_corr).
//
// With WAVE != 0, the warp takes the rows wave_row0, wave_row0 + wave_stride, ... below
// wave_end instead of a grid stride, and X and Z are read with
// coherent loads (WAVE 1: ld.global.cg, L2 only, so no L1 line can hold a stale
// copy; WAVE 2: plain loads; WAVE 3: the read-only path, for launches that run one
// step): the multi-step filter (cheb_wave_kernel) reads blocks that other CTAs of the
// same launch wrote.
// Cross-level link of the multi-step filter (cheb_wave_kernel): the level this warp
// runs waits, before each row, until the previous level has finished every row up
// to `reach` past it, and reports each finished row. Rows are counted per block of
// 2^block_shift rows.
struct WaveLink {
  const int* prev_done;  // finished-row counts of the previous level (null: no wait)
  int* own_done;         // this level's counts
  int64_t reach;         // operator bandwidth
  int64_t nrows;
  int block_shift;
  const int* abort_flag;
  int* status;
  long long max_polls;
  int64_t* known;  // this warp's count of leading blocks known complete (shared memory)
};

constexpr int kWaveTimeoutCode = 13;

__device__ __forceinline__ int ld_acquire_s32(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Returns false if the wait timed out or the launch was aborted (the warp stops).
__device__ __forceinline__ bool wave_wait(const WaveLink& L, int64_t row) {
  const int lane = threadIdx.x & 31;
  const int64_t need_row = min(L.nrows - 1, row + L.reach);
  const int64_t need = need_row >> L.block_shift;  // blocks [0, need] must be complete
  int64_t known = *L.known;
  if (known > need) return true;
  const int64_t nblocks = ((L.nrows - 1) >> L.block_shift) + 1;
  const int64_t brows = int64_t(1) << L.block_shift;
  long long polls = 0;
  while (true) {
    const int64_t b = known + lane;
    int f = 1;
    if (b < nblocks) {
      const int64_t full = min(brows, L.nrows - b * brows);
      f = ld_acquire_s32(L.prev_done + b) == full;
    }
    const unsigned m = __ballot_sync(0xffffffffu, f != 0);
    known += m == 0xffffffffu ? 32 : __ffs(~m) - 1;
    if (known > need) break;
    if (m != 0xffffffffu) {
      int halt = 0;
      if (lane == 0) {
        halt = *reinterpret_cast<const volatile int*>(L.abort_flag) != 0;
        if (!halt && ++polls > L.max_polls) {
          atomicCAS(L.status ? L.status : &g_spmm_status, 0, kWaveTimeoutCode);
          atomicExch(const_cast<int*>(L.abort_flag), 1);
          halt = 1;
        }
      }
      if (__shfl_sync(0xffffffffu, halt, 0)) return false;
      __nanosleep(64);
    }
  }
  if (lane == 0) *L.known = known;
  __syncwarp();
  return true;
}

// Finished rows are reported kWaveBatch at a time: one fence per batch (a fence waits
// for the warp's stores to drain, which stalls a latency-bound warp), then relaxed
// increments of the batch's block counters. `pending` holds the batch's rows.
constexpr int kWaveBatch = 4;

__device__ __forceinline__ void wave_flush(const WaveLink& L, const int64_t (&pending)[kWaveBatch],
                                           int count) {
  __syncwarp();  // every lane's stores precede the fence below
  if ((threadIdx.x & 31) == 0 && count > 0) {
    __threadfence();
#pragma unroll
    for (int i = 0; i < kWaveBatch; ++i)
      if (i < count)
        asm volatile("red.relaxed.gpu.global.add.s32 [%0], 1;" ::"l"(
                         L.own_done + (pending[i] >> L.block_shift))
                     : "memory");
  }
}

__device__ __forceinline__ void wave_done(const WaveLink& L, int64_t row,
                                          int64_t (&pending)[kWaveBatch], int& count) {
  if (!L.own_done) return;  // the last level of a launch: nobody waits on it
#pragma unroll
  for (int i = 0; i < kWaveBatch; ++i)
    if (i == count) pending[i] = row;
  if (++count == kWaveBatch) {
    wave_flush(L, pending, count);
    count = 0;
  }
}

// X loads of the row body: WAVE 0 and 3 = read-only path (X not written during the
// launch), 1 = L2 only (ld.global.cg), 2 = plain coherent loads.
template <typename T, int VEC, int WAVE>
__device__ __forceinline__ Pack<T, VEC> body_load_x(const T* p) {
  if constexpr (WAVE == 1) return load_pack_cg<T, VEC>(p);
  else if constexpr (WAVE == 2) return load_pack_rw<T, VEC>(p);
  else return load_pack<T, VEC>(p);
}

template <typename T, int VEC, int CPL, int NZ, bool CORR, int WAVE = 0, int XL = -1>
__device__ __forceinline__ void csr_spmm_row_body(
    int64_t nrows, const int32_t* __restrict__ rowptr, const int32_t* __restrict__ colind,
    const T* __restrict__ vals, const T* X, int64_t ldx, T* Y, int64_t ldy,
    const T* Z, int64_t ldz, int ncols, int panel_vec, T alpha, T gamma, T beta, int use_gamma,
    int use_beta, int prefetch_z, const T* __restrict__ R, int64_t ldr,
    const T* __restrict__ delta, int64_t wave_row0 = 0, int64_t wave_end = 0,
    int64_t wave_stride = 1, const WaveLink* link = nullptr) {
  constexpr unsigned kFull = 0xffffffffu;
  // load kind of X and Z: XL if given, else by the wave mode (see body_load_x)
  constexpr int XLK = XL >= 0 ? XL : WAVE;
  const int lane = threadIdx.x & 31;
  const int64_t tw = WAVE != 0 ? wave_stride : static_cast<int64_t>(gridDim.x) * (kThreads / 32);
  int64_t row = WAVE != 0 ? wave_row0
                          : static_cast<int64_t>(blockIdx.x) * (kThreads / 32) + threadIdx.x / 32;
  const int64_t row_end = WAVE != 0 ? wave_end : nrows;
  if (row >= row_end) return;
  const int p0 = blockIdx.y * panel_vec * VEC;
  const int nvec = min(panel_vec, (ncols - p0) / VEC);
  const T* Xp = X + p0;

  int s0 = __ldg(rowptr + row), e0 = __ldg(rowptr + row + 1);
  int c_cur = 0;
  T a_cur = T(0);
  if (lane < min(e0 - s0, NZ)) {
    c_cur = __ldg(colind + s0 + lane);
    a_cur = __ldg(vals + s0 + lane);
  }
  int64_t nxt = row + tw;
  int s1 = 0, e1 = 0;
  if (nxt < row_end) {
    s1 = __ldg(rowptr + nxt);
    e1 = __ldg(rowptr + nxt + 1);
  }
  int64_t pending[kWaveBatch];
  int npending = 0;
  while (true) {
    if constexpr (WAVE != 0) {
      if (link->prev_done) {
        const int64_t need = min(link->nrows - 1, row + link->reach) >> link->block_shift;
        if (*link->known <= need) {
          // about to wait: report this warp's finished rows first
          if (link->own_done && npending > 0) {
            wave_flush(*link, pending, npending);
            npending = 0;
          }
          if (!wave_wait(*link, row)) return;
        }
      }
    }
    const int nnz = e0 - s0;
    Pack<T, VEC> z[CPL];
    Pack<T, VEC> rc[CPL];
    if constexpr (CORR) {
#pragma unroll
      for (int q = 0; q < CPL; ++q) {
        const int v = lane + 32 * q;
        if (v < nvec) rc[q] = load_pack_rw<T, VEC>(R + row * ldr + p0 + v * VEC);
      }
    }
    if (use_beta) {
#pragma unroll
      for (int q = 0; q < CPL; ++q) {
        const int v = lane + 32 * q;
        if (v < nvec)
          z[q] = XLK == 1 ? load_pack_cg<T, VEC>(Z + row * ldz + p0 + v * VEC)
                          : load_pack_rw<T, VEC>(Z + row * ldz + p0 + v * VEC);
      }
      // Z rows stream from DRAM: with prefetch_z, start this warp's next Z row
      // toward L2 now (one 128-byte line per lane, addresses inside the row), so
      // its loads there meet L2 rather than DRAM latency (pays off for the FP64
      // panels, not for one FP32 panel: a per-operator autotune choice).
      if (prefetch_z && nxt < row_end) {
        const int bytes = nvec * VEC * static_cast<int>(sizeof(T));
        if (lane * 128 < bytes)
          asm volatile("prefetch.global.L2 [%0];" ::"l"(
              reinterpret_cast<const char*>(Z + nxt * ldz + p0) + lane * 128));
        // The next row's farthest neighbour, guessed by translating this row's
        // (exact for a translation-invariant stencil; a wrong guess only wastes
        // the prefetch): the X row a banded operator touches first.
        const int cl = __shfl_sync(kFull, c_cur, min(nnz, NZ) - 1);
        const int64_t cg = cl + (nxt - row);
        if (nnz > 0 && cg >= 0 && cg < nrows && lane >= 16 && (lane - 16) * 128 < bytes)
          asm volatile("prefetch.global.L2 [%0];" ::"l"(
              reinterpret_cast<const char*>(Xp + cg * ldx) + (lane - 16) * 128));
      }
    }
    T acc[CPL][VEC];
#pragma unroll
    for (int q = 0; q < CPL; ++q)
#pragma unroll
      for (int e = 0; e < VEC; ++e) acc[q][e] = T(0);
    bool self_found = false;
    // next-row metadata, prefetched under this row's loads
    int c_n = 0;
    T a_n = T(0);
    int64_t nxt2 = nxt + tw;
    int s2 = 0, e2 = 0;
    if (nnz <= NZ) {
      Pack<T, VEC> x[NZ][CPL];
#pragma unroll
      for (int t = 0; t < NZ; ++t) {
        const int c = __shfl_sync(kFull, c_cur, t);
        if (t < nnz) {
          const T* xr = Xp + static_cast<int64_t>(c) * ldx;
#pragma unroll
          for (int q = 0; q < CPL; ++q) {
            const int v = lane + 32 * q;
            if (v < nvec) x[t][q] = body_load_x<T, VEC, XLK>(xr + v * VEC);
          }
        }
      }
      if (nxt < row_end && lane < min(e1 - s1, NZ)) {
        c_n = __ldg(colind + s1 + lane);
        a_n = __ldg(vals + s1 + lane);
      }
      if (nxt2 < row_end) {
        s2 = __ldg(rowptr + nxt2);
        e2 = __ldg(rowptr + nxt2 + 1);
      }
#pragma unroll
      for (int t = 0; t < NZ; ++t) {
        const int c = __shfl_sync(kFull, c_cur, t);
        T coef = alpha * __shfl_sync(kFull, a_cur, t);
        if (t < nnz) {
          if (c == row) {
            coef += gamma;
            self_found = true;
          }
#pragma unroll
          for (int q = 0; q < CPL; ++q) {
            const int v = lane + 32 * q;
            if (v < nvec) {
#pragma unroll
              for (int e = 0; e < VEC; ++e) acc[q][e] = fma(coef, x[t][q].v[e], acc[q][e]);
            }
          }
        }
      }
    } else {
      // Long row: stream its nonzeros 32 at a time.
      for (int base = s0; base < e0; base += 32) {
        const int k = base + lane;
        int c = 0;
        T a = T(0);
        if (k < e0) {
          c = __ldg(colind + k);
          a = __ldg(vals + k);
        }
        const int cnt = min(32, e0 - base);
        for (int t = 0; t < cnt; ++t) {
          const int c0 = __shfl_sync(kFull, c, t);
          T coef = alpha * __shfl_sync(kFull, a, t);
          if (c0 == row) {
            coef += gamma;
            self_found = true;
          }
          const T* xr = Xp + static_cast<int64_t>(c0) * ldx;
#pragma unroll
          for (int q = 0; q < CPL; ++q) {
            const int v = lane + 32 * q;
            if (v < nvec) {
              const Pack<T, VEC> p = body_load_x<T, VEC, XLK>(xr + v * VEC);
#pragma unroll
              for (int e = 0; e < VEC; ++e) acc[q][e] = fma(coef, p.v[e], acc[q][e]);
            }
          }
        }
      }
      if (nxt < row_end && lane < min(e1 - s1, NZ)) {
        c_n = __ldg(colind + s1 + lane);
        a_n = __ldg(vals + s1 + lane);
      }
      if (nxt2 < row_end) {
        s2 = __ldg(rowptr + nxt2);
        e2 = __ldg(rowptr + nxt2 + 1);
      }
    }
    if (use_gamma && !self_found) {
#pragma unroll
      for (int q = 0; q < CPL; ++q) {
        const int v = lane + 32 * q;
        if (v < nvec) {
          const Pack<T, VEC> xr = body_load_x<T, VEC, XLK>(Xp + row * ldx + v * VEC);
#pragma unroll
          for (int e = 0; e < VEC; ++e) acc[q][e] = fma(gamma, xr.v[e], acc[q][e]);
        }
      }
    }
    T* yr = Y + row * ldy + p0;
#pragma unroll
    for (int q = 0; q < CPL; ++q) {
      const int v = lane + 32 * q;
      if (v < nvec) {
        Pack<T, VEC> out;
#pragma unroll
        for (int e = 0; e < VEC; ++e)
          out.v[e] = use_beta ? fma(beta, z[q].v[e], acc[q][e]) : acc[q][e];
        if constexpr (CORR) {
          const Pack<T, VEC> dl = load_pack<T, VEC>(delta + p0 + v * VEC);
#pragma unroll
          for (int e = 0; e < VEC; ++e) out.v[e] = fma(dl.v[e], rc[q].v[e], out.v[e]);
        }
        store_pack<T, VEC>(yr + v * VEC, out);
      }
    }
    if constexpr (WAVE != 0) wave_done(*link, row, pending, npending);
    if (nxt >= row_end) break;
    row = nxt;
    nxt = nxt2;
    s0 = s1;
    e0 = e1;
    s1 = s2;
    e1 = e2;
    c_cur = c_n;
    a_cur = a_n;
  }
  if constexpr (WAVE != 0) {
    if (link->own_done) wave_flush(*link, pending, npending);
  }
}

template <typename T, int VEC, int CPL, int NZ>
__global__ void __launch_bounds__(kThreads)
csr_spmm_row_kernel(int64_t nrows, const int32_t* __restrict__ rowptr,
                    const int32_t* __restrict__ colind, const T* __restrict__ vals,
                    const T* __restrict__ X, int64_t ldx, T* Y, int64_t ldy, const T* Z,
                    int64_t ldz, int ncols, int panel_vec, T alpha, T gamma, T beta,
                    int use_gamma, int use_beta, int prefetch_z) {
  csr_spmm_row_body<T, VEC, CPL, NZ, false>(nrows, rowptr, colind, vals, X, ldx, Y, ldy, Z, ldz,
                                            ncols, panel_vec, alpha, gamma, beta, use_gamma,
                                            use_beta, prefetch_z, nullptr, 0, nullptr);
}

// The row kernel with X and Z read through L2 only (ld.global.cg): gathers whose
// neighbour rows see little L1 reuse skip the L1 allocation (SpMM mode 7).
template <typename T, int VEC, int CPL, int NZ>
__global__ void __launch_bounds__(kThreads)
csr_spmm_row_cg_kernel(int64_t nrows, const int32_t* __restrict__ rowptr,
                       const int32_t* __restrict__ colind, const T* __restrict__ vals,
                       const T* __restrict__ X, int64_t ldx, T* Y, int64_t ldy, const T* Z,
                       int64_t ldz, int ncols, int panel_vec, T alpha, T gamma, T beta,
                       int use_gamma, int use_beta, int prefetch_z) {
  csr_spmm_row_body<T, VEC, CPL, NZ, false, 0, 1>(nrows, rowptr, colind, vals, X, ldx, Y, ldy, Z,
                                                  ldz, ncols, panel_vec, alpha, gamma, beta,
                                                  use_gamma, use_beta, prefetch_z, nullptr, 0,
                                                  nullptr);
}

// The row kernel with the correction term delta[j] * R[row, j] added to every output
// (the refined filter's recurrence, csr_spmm_corr_f32); register use bounded for two
// CTAs per SM.
template <typename T, int VEC, int CPL, int NZ>
__global__ void __launch_bounds__(kThreads, 2)
csr_spmm_row_corr_kernel(int64_t nrows, const int32_t* __restrict__ rowptr,
                         const int32_t* __restrict__ colind, const T* __restrict__ vals,
                         const T* __restrict__ X, int64_t ldx, T* Y, int64_t ldy, const T* Z,
                         int64_t ldz, int ncols, int panel_vec, T alpha, T gamma, T beta,
                         int use_gamma, int use_beta, const T* __restrict__ R, int64_t ldr,
                         const T* __restrict__ delta) {
  csr_spmm_row_body<T, VEC, CPL, NZ, true>(nrows, rowptr, colind, vals, X, ldx, Y, ldy, Z, ldz,
                                           ncols, panel_vec, alpha, gamma, beta, use_gamma,
                                           use_beta, 0, R, ldr, delta);
}

// ---------------------------------------------------------------------------
// Multi-step Chebyshev filter in one launch (levels trailing each other over rows).
//
// Step k of the filter writes Y_k = alpha_k A Y_{k-1} + gamma_k Y_{k-1} + beta_k Y_{k-2}
// into the buffer that held Y_{k-2} (buf[k & 1]; buf[0] holds the input block). Row r
// of Y_k needs the rows of Y_{k-1} within the operator's bandwidth bw of r. One
// launch runs `levels` consecutive steps: the warps of the grid are dealt round-robin
// to the levels, and the warps of a level sweep the rows exactly as the single-step
// row kernel does (warp j of the level: rows j, j + W, j + 2W, ..., W the level's
// warps), so each level's rows in flight stay within a narrow band. Before each row,
// a warp of level k waits until level k - 1 has finished every row up to bw past it
// (finished rows are counted per block of 1024 rows with release increments and read
// with acquire loads), so level k runs about bw rows behind level k - 1 and gathers
// rows of Y_{k-1} written a moment before, from L2. A launch of S steps therefore
// reads two blocks from DRAM and writes S, where S single steps read 2 S and write S.
// In-place overwrites are safe: level k overwrites row r of Y_{k-2} only after level
// k - 1, the last reader of those rows near r, has passed r + bw. The first level
// never waits and every level waits only on the one before, so with all warps
// resident (a cooperative launch) the schedule cannot deadlock; every wait is
// bounded (timeout: status code 13 and an abort flag that stops every waiting warp).
// The arithmetic of every row is that of the single-step row kernel (bit-identical
// results). Blocks are read with ld.global.cg (L2 only): rows are rewritten by other
// SMs during the launch, and no L1 line may hold a stale copy.
constexpr int kWaveMaxLevels = 8;
constexpr int kWaveBlockShift = 10;  // 1024 rows per completion counter

template <typename T>
struct WaveParams {
  int64_t nrows;
  const int32_t* rowptr;
  const int32_t* colind;
  const T* vals;
  T* buf[2];
  int64_t ld[2];
  int ncols, panel_vec;
  int levels;   // steps in this launch
  int first_k;  // filter step of level 0 (1-based)
  T alpha[kWaveMaxLevels], gamma[kWaveMaxLevels], beta[kWaveMaxLevels];
  int64_t reach;  // operator bandwidth (rows)
  int* done;      // levels x blocks finished-row counters
  int64_t nblocks;
  int* abort_flag;
  int* status;
  long long max_polls;
};

template <typename T, int VEC, int CPL, int NZ, int LOADS>
__global__ void __launch_bounds__(kThreads, 2)
cheb_wave_kernel(const __grid_constant__ WaveParams<T> P) {
  static_assert(LOADS >= 1 && LOADS <= 3, "the multi-step kernel sweeps rows per level");
  __shared__ int64_t s_known[kThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) s_known[warp] = 0;
  __syncwarp();
  const int64_t gw = static_cast<int64_t>(blockIdx.x) * (kThreads / 32) + warp;
  const int64_t nw = static_cast<int64_t>(gridDim.x) * (kThreads / 32);
  const int lev = static_cast<int>(gw % P.levels);
  const int64_t j = gw / P.levels;
  const int64_t wl = (nw - lev + P.levels - 1) / P.levels;  // warps of this level
  WaveLink L;
  L.prev_done = lev > 0 ? P.done + static_cast<int64_t>(lev - 1) * P.nblocks : nullptr;
  L.own_done = lev + 1 < P.levels ? P.done + static_cast<int64_t>(lev) * P.nblocks : nullptr;
  L.reach = P.reach;
  L.nrows = P.nrows;
  L.block_shift = kWaveBlockShift;
  L.abort_flag = P.abort_flag;
  L.status = P.status;
  L.max_polls = P.max_polls;
  L.known = &s_known[warp];
  const int k = P.first_k + lev;
  T* out = P.buf[k & 1];
  const int64_t ldo = P.ld[k & 1];
  const T* cur = P.buf[(k - 1) & 1];
  const int64_t ldc = P.ld[(k - 1) & 1];
  const T be = P.beta[lev];
  csr_spmm_row_body<T, VEC, CPL, NZ, false, LOADS>(
      P.nrows, P.rowptr, P.colind, P.vals, cur, ldc, out, ldo, out, ldo, P.ncols, P.panel_vec,
      P.alpha[lev], P.gamma[lev], be, 1, be != T(0) ? 1 : 0, 0, nullptr, 0, nullptr, j, P.nrows,
      wl, &L);
}

template <typename T, int VEC>
bool try_row_kernel(const Csr& A, const T* vals, const T* X, int64_t ldx, T* Y, int64_t ldy,
                    const T* Z, int64_t ldz, int ncols, T alpha, T gamma, T beta, bool ug, bool ub,
                    cudaStream_t s, int max_cpl, bool prefetch_z = false, bool cg = false) {
  constexpr int NZ = 7;
  const int nvec = ncols / VEC;
  if (nvec < 32 || ncols % VEC != 0 || A.max_row_nnz > NZ) return false;
  const int panels = (nvec + 32 * max_cpl - 1) / (32 * max_cpl);
  const int panel_vec = (nvec + panels - 1) / panels;
  const int cpl = (panel_vec + 31) / 32;
  // One warp per row, grid-stride over rows with exactly the resident CTAs.
#define FE_ROW(CPL_)                                                                           \
  do {                                                                                         \
    auto kern = cg ? csr_spmm_row_cg_kernel<T, VEC, CPL_, NZ>                                  \
                   : csr_spmm_row_kernel<T, VEC, CPL_, NZ>;                                    \
    static int resident_by_kind[2] = {0, 0};                                                   \
    int& resident = resident_by_kind[cg ? 1 : 0];                                              \
    if (resident == 0) {                                                                       \
      FE_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, kern, kThreads,   \
                                                                  0));                         \
      resident = std::max(resident, 1);                                                        \
    }                                                                                          \
    int64_t blocks = std::min<int64_t>((A.rows + 7) / 8,                                       \
                                       static_cast<int64_t>(num_sms()) * resident);            \
    blocks = std::max<int64_t>(blocks, 1);                                                     \
    dim3 grid(static_cast<unsigned>(blocks), static_cast<unsigned>(panels));                   \
    kern<<<grid, kThreads, 0, s>>>(A.rows, A.rowptr, A.colind, vals, X, ldx, Y, ldy, Z, ldz,   \
                                   ncols, panel_vec, alpha, gamma, beta, ug ? 1 : 0,           \
                                   ub ? 1 : 0, prefetch_z && A.rows == A.cols ? 1 : 0);        \
    check_launch("csr_spmm_row_kernel");                                                       \
  } while (0)
  if (cpl == 1) FE_ROW(1);
  else if (cpl == 2) FE_ROW(2);
  else if (cpl == 3) FE_ROW(3);
  else if (cpl == 4) FE_ROW(4);
  else FE_ROW(5);
#undef FE_ROW
  return true;
}

// Y[:, j] += delta[j] * R[:, j] (the correction term where the row kernel does not
// apply).
__global__ void col_scaled_add_kernel(int64_t n, int ncols, const float* __restrict__ R,
                                      int64_t ldr, const float* __restrict__ delta,
                                      float* __restrict__ Y, int64_t ldy) {
  const int64_t total = n * ncols;
  for (int64_t idx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; idx < total;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i = idx / ncols;
    const int j = static_cast<int>(idx % ncols);
    Y[i * ldy + j] = fmaf(delta[j], R[i * ldr + j], Y[i * ldy + j]);
  }
}

// Start of the refined filter: R32 = float(R64 - theta_j X) and Z1 = c * R32.
__global__ void refine_start_kernel(int64_t n, int ncols, const double* __restrict__ R64,
                                    int64_t ld64, const double* __restrict__ X, int64_t ldx,
                                    const double* __restrict__ theta, double c,
                                    float* __restrict__ R32, float* __restrict__ Z1,
                                    int64_t ld32) {
  const int64_t total = n * ncols;
  for (int64_t idx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; idx < total;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i = idx / ncols;
    const int j = static_cast<int>(idx % ncols);
    const double r = R64[i * ld64 + j] - theta[j] * X[i * ldx + j];
    R32[i * ld32 + j] = static_cast<float>(r);
    Z1[i * ld32 + j] = static_cast<float>(c * r);
  }
}

// End of the refined filter: X = t_j X + Z (FP64).
__global__ void refine_finish_kernel(int64_t n, int ncols, const double* __restrict__ t,
                                     const float* __restrict__ Z, int64_t ld32,
                                     double* __restrict__ X, int64_t ldx) {
  const int64_t total = n * ncols;
  for (int64_t idx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; idx < total;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i = idx / ncols;
    const int j = static_cast<int>(idx % ncols);
    X[i * ldx + j] = fma(t[j], X[i * ldx + j], static_cast<double>(Z[i * ld32 + j]));
  }
}

inline unsigned elementwise_grid(int64_t total) {
  return static_cast<unsigned>(std::min<int64_t>((total + 255) / 256, int64_t(148) * 32));
}

template <typename T, int VEC, int G, int CPL>
void launch_one(const Csr& A, const T* vals, const T* X, int64_t ldx, T* Y, int64_t ldy,
                const T* Z, int64_t ldz, int ncols, T alpha, T gamma, T beta, bool ug,
                bool ub, cudaStream_t s) {
  constexpr int rows_per_block = kThreads / G;
  const int64_t blocks = (A.rows + rows_per_block - 1) / rows_per_block;
  const int panel = G * CPL * VEC;
  const int panels = (ncols + panel - 1) / panel;
  FE_REQUIRE(blocks <= 0x7fffffffLL, "csr_spmm: too many rows for one launch");
  dim3 grid(static_cast<unsigned>(blocks), static_cast<unsigned>(panels));
  csr_spmm_kernel<T, VEC, G, CPL><<<grid, kThreads, 0, s>>>(
      A.rows, A.rowptr, A.colind, vals, X, ldx, Y, ldy, Z, ldz, ncols, alpha, gamma, beta,
      ug ? 1 : 0, ub ? 1 : 0);
  check_launch("csr_spmm_kernel");
}

template <typename T, int VEC>
void dispatch_vec(const Csr& A, const T* vals, const T* X, int64_t ldx, T* Y, int64_t ldy,
                  const T* Z, int64_t ldz, int ncols, T alpha, T gamma, T beta, bool ug,
                  bool ub, cudaStream_t s) {
  const int nvec = (ncols + VEC - 1) / VEC;
#define FE_LAUNCH(G_, CPL_) \
  launch_one<T, VEC, G_, CPL_>(A, vals, X, ldx, Y, ldy, Z, ldz, ncols, alpha, gamma, beta, ug, ub, s)
  if (nvec <= 1) FE_LAUNCH(1, 1);
  else if (nvec <= 2) FE_LAUNCH(2, 1);
  else if (nvec <= 4) FE_LAUNCH(4, 1);
  else if (nvec <= 8) FE_LAUNCH(8, 1);
  else if (nvec <= 16) FE_LAUNCH(16, 1);
  else if (nvec <= 32) FE_LAUNCH(32, 1);
  else if (nvec <= 64) FE_LAUNCH(32, 2);
  else if (nvec <= 96) FE_LAUNCH(32, 3);
  else if (nvec <= 128) FE_LAUNCH(32, 4);
  else if (nvec <= 160) FE_LAUNCH(32, 5);
  else if (nvec <= 192) FE_LAUNCH(32, 6);
  else FE_LAUNCH(32, 8);  // wider blocks run as column panels of 256 vectors
#undef FE_LAUNCH
}

// ---------------------------------------------------------------------------
// Bulk-copy pipelined SpMM (the path for matrices whose rows have at most a
// few tens of nonzeros, e.g. the 7-, 13- and 27-point stencils).
//
// One warp owns a sequence of rows (row = global_warp + i * total_warps) and
// keeps kPipeDepth rows in flight: for the next rows it issues one
// cp.async.bulk (TMA bulk copy, 16-byte aligned, no registers held) per nonzero
// to gather the neighbour rows of X, plus one for the Z row, into a per-warp
// shared-memory stage tracked by an mbarrier with a transaction count. While
// those copies land, the warp accumulates the previous row from shared memory.
// This removes the chain of dependent global loads per row that bounds the
// register-only kernel and keeps ~128 KB per SM in flight.
// ---------------------------------------------------------------------------
constexpr int kPipeWarps = 8;
constexpr int kPipeDepth = 2;
constexpr int kPipeMaxSlots = 32;
constexpr int kPipeStageBytes = 10240;  // per warp and stage: slots * row bytes

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void pipe_bar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)));
}

__device__ __forceinline__ void pipe_arrive_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool pipe_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait (about two seconds of SM clock); records `code` on timeout.
__device__ __forceinline__ bool pipe_wait(uint64_t* bar, uint32_t parity, int code, int* status) {
  if (pipe_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (true) {
    for (int i = 0; i < 64; ++i)
      if (pipe_try_wait(bar, parity)) return true;
    if (clock64() - t0 > 4000000000LL) {
      atomicCAS(status ? status : &g_spmm_status, 0, code);
      return false;
    }
  }
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

template <typename T>
struct PipeLayout {
  uint64_t* bars;   // [warps][depth]
  int32_t* nnz;     // [warps][depth]
  int32_t* cols;    // [warps][depth][kPipeMaxSlots]
  T* vals;          // [warps][depth][kPipeMaxSlots]
  uint8_t* data;    // [warps][depth][slots][row_bytes]
};

template <typename T>
__device__ __forceinline__ PipeLayout<T> pipe_layout(uint8_t* smem) {
  PipeLayout<T> L;
  L.bars = reinterpret_cast<uint64_t*>(smem);
  L.nnz = reinterpret_cast<int32_t*>(smem + kPipeWarps * kPipeDepth * 8);
  L.cols = L.nnz + kPipeWarps * kPipeDepth;
  L.vals = reinterpret_cast<T*>(L.cols + kPipeWarps * kPipeDepth * kPipeMaxSlots);
  uintptr_t d = reinterpret_cast<uintptr_t>(L.vals + kPipeWarps * kPipeDepth * kPipeMaxSlots);
  d = (d + 127) & ~uintptr_t(127);
  L.data = reinterpret_cast<uint8_t*>(d);
  return L;
}

template <typename T>
constexpr size_t pipe_smem_bytes() {
  return kPipeWarps * kPipeDepth * (8 + 4 + kPipeMaxSlots * (4 + sizeof(T))) + 128 +
         static_cast<size_t>(kPipeWarps) * kPipeDepth * kPipeStageBytes;
}

template <typename T, int VEC, int CPL>
__global__ void __launch_bounds__(kPipeWarps * 32, 1)
csr_spmm_pipe_kernel(int64_t nrows, const int32_t* __restrict__ rowptr,
                     const int32_t* __restrict__ colind, const T* __restrict__ vals,
                     const T* __restrict__ X, int64_t ldx, T* Y, int64_t ldy, const T* Z,
                     int64_t ldz, int ncols, int panel_cols, int slots, T alpha, T gamma, T beta,
                     int use_gamma, int use_beta, int* status) {
  extern __shared__ __align__(128) uint8_t pipe_smem[];
  const PipeLayout<T> L = pipe_layout<T>(pipe_smem);
  const int warp = threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  const int panel0 = blockIdx.y * panel_cols;
  const int width = min(panel_cols, ncols - panel0);
  const uint32_t row_bytes = static_cast<uint32_t>(width) * sizeof(T);
  const int nvec = width / VEC;
  const int64_t gwarp = static_cast<int64_t>(blockIdx.x) * kPipeWarps + warp;
  const int64_t twarps = static_cast<int64_t>(gridDim.x) * kPipeWarps;

  uint64_t* bars = L.bars + warp * kPipeDepth;
  int32_t* m_nnz = L.nnz + warp * kPipeDepth;
  int32_t* m_cols = L.cols + warp * kPipeDepth * kPipeMaxSlots;
  T* m_vals = L.vals + warp * kPipeDepth * kPipeMaxSlots;
  uint8_t* m_data = L.data + static_cast<size_t>(warp) * kPipeDepth * kPipeStageBytes;

  if (lane == 0) {
    for (int s = 0; s < kPipeDepth; ++s) pipe_bar_init(&bars[s]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncwarp();

  // Gather row r's neighbour rows (and its Z row) into stage s.
  auto issue = [&](int64_t r, int s) {
    const int start = __ldg(rowptr + r);
    const int nnz = __ldg(rowptr + r + 1) - start;
    uint8_t* stage = m_data + s * kPipeStageBytes;
    if (nnz > slots - 1) {  // too many neighbours: the consumer reads them directly
      if (lane == 0) {
        m_nnz[s] = -1;
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&bars[s]))
                     : "memory");
      }
      __syncwarp();
      return;
    }
    int c = 0;
    if (lane < nnz) {
      c = __ldg(colind + start + lane);
      m_cols[s * kPipeMaxSlots + lane] = c;
      m_vals[s * kPipeMaxSlots + lane] = __ldg(vals + start + lane);
    }
    if (lane == 0) {
      m_nnz[s] = nnz;
      pipe_arrive_tx(&bars[s], static_cast<uint32_t>(nnz + use_beta) * row_bytes);
    }
    __syncwarp();
    if (lane < nnz) bulk_g2s(stage + lane * row_bytes, X + static_cast<int64_t>(c) * ldx + panel0,
                             row_bytes, &bars[s]);
    if (use_beta && lane == 31)
      bulk_g2s(stage + (slots - 1) * row_bytes, Z + r * ldz + panel0, row_bytes, &bars[s]);
  };

  for (int s = 0; s < kPipeDepth; ++s) {
    const int64_t r = gwarp + s * twarps;
    if (r < nrows) issue(r, s);
  }

  bool ok = true;
  for (int64_t i = 0;; ++i) {
    const int64_t r = gwarp + i * twarps;
    if (r >= nrows) break;
    const int s = static_cast<int>(i % kPipeDepth);
    const uint32_t parity = static_cast<uint32_t>((i / kPipeDepth) & 1);
    if (!pipe_wait(&bars[s], parity, 11, status)) {
      ok = false;
      break;
    }
    const int nnz = m_nnz[s];
    const uint8_t* stage = m_data + s * kPipeStageBytes;
    T acc[CPL][VEC];
#pragma unroll
    for (int q = 0; q < CPL; ++q)
#pragma unroll
      for (int e = 0; e < VEC; ++e) acc[q][e] = T(0);
    int self_slot = -1;
    if (nnz >= 0) {
      for (int k = 0; k < nnz; ++k) {
        const T a = m_vals[s * kPipeMaxSlots + k];
        if (m_cols[s * kPipeMaxSlots + k] == r) self_slot = k;
        const T* xs = reinterpret_cast<const T*>(stage + k * row_bytes);
#pragma unroll
        for (int q = 0; q < CPL; ++q) {
          const int v = lane + q * 32;
          if (v < nvec) {
            const Pack<T, VEC> p = load_pack_rw<T, VEC>(xs + v * VEC);
#pragma unroll
            for (int e = 0; e < VEC; ++e) acc[q][e] = fma(a, p.v[e], acc[q][e]);
          }
        }
      }
    } else {
      const int start = __ldg(rowptr + r);
      const int end = __ldg(rowptr + r + 1);
      for (int base = start; base < end; base += 32) {
        const int k = base + lane;
        int c = 0;
        T a = T(0);
        if (k < end) {
          c = __ldg(colind + k);
          a = __ldg(vals + k);
        }
        const int cnt = min(32, end - base);
        for (int t = 0; t < cnt; ++t) {
          const int c0 = __shfl_sync(0xffffffffu, c, t);
          const T a0 = __shfl_sync(0xffffffffu, a, t);
          const T* x0 = X + static_cast<int64_t>(c0) * ldx + panel0;
#pragma unroll
          for (int q = 0; q < CPL; ++q) {
            const int v = lane + q * 32;
            if (v < nvec) {
              const Pack<T, VEC> p = load_pack<T, VEC>(x0 + v * VEC);
#pragma unroll
              for (int e = 0; e < VEC; ++e) acc[q][e] = fma(a0, p.v[e], acc[q][e]);
            }
          }
        }
      }
    }
    const T* xself = (self_slot >= 0)
                         ? reinterpret_cast<const T*>(stage + self_slot * row_bytes)
                         : X + r * ldx + panel0;
    const T* zrow = (nnz >= 0) ? reinterpret_cast<const T*>(stage + (slots - 1) * row_bytes)
                               : Z + r * ldz + panel0;
    T* yrow = Y + r * ldy + panel0;
#pragma unroll
    for (int q = 0; q < CPL; ++q) {
      const int v = lane + q * 32;
      if (v < nvec) {
        Pack<T, VEC> out;
#pragma unroll
        for (int e = 0; e < VEC; ++e) out.v[e] = alpha * acc[q][e];
        if (use_gamma) {
          const Pack<T, VEC> xr = load_pack_rw<T, VEC>(xself + v * VEC);
#pragma unroll
          for (int e = 0; e < VEC; ++e) out.v[e] = fma(gamma, xr.v[e], out.v[e]);
        }
        if (use_beta) {
          const Pack<T, VEC> zr = load_pack_rw<T, VEC>(zrow + v * VEC);
#pragma unroll
          for (int e = 0; e < VEC; ++e) out.v[e] = fma(beta, zr.v[e], out.v[e]);
        }
        store_pack<T, VEC>(yrow + v * VEC, out);
      }
    }
    __syncwarp();
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    const int64_t rn = gwarp + (i + kPipeDepth) * twarps;
    if (rn < nrows) issue(rn, s);
  }
  if (!ok) {
    // Let copies already issued for this warp land before the CTA exits.
    for (int s = 0; s < kPipeDepth; ++s) pipe_wait(&bars[s], 0, 12, status);
  }
}

template <typename T, int VEC>
bool try_pipe(const Csr& A, const T* vals, const T* X, int64_t ldx, T* Y, int64_t ldy, const T* Z,
              int64_t ldz, int ncols, T alpha, T gamma, T beta, bool ug, bool ub, cudaStream_t s) {
  // Panel width: the widest multiple of 32 vectors whose rows fit the stage
  // with one slot per neighbour plus the Z row.
  const int need_slots = static_cast<int>(A.max_row_nnz) + 1;
  if (need_slots > kPipeMaxSlots) return false;
  const int max_row_bytes = (kPipeStageBytes / need_slots) & ~15;
  int panel = std::min(ncols, max_row_bytes / static_cast<int>(sizeof(T)));
  panel = std::min(panel, 8 * 32 * VEC);  // CPL <= 8
  if (panel < VEC || panel * static_cast<int>(sizeof(T)) % 16 != 0) return false;
  if (panel < ncols) panel = (panel / (32 * VEC)) * 32 * VEC;  // full-warp panels when split
  if (panel <= 0 || (ncols % panel) * sizeof(T) % 16 != 0) return false;
  const int slots = std::min(kPipeMaxSlots, kPipeStageBytes / (panel * static_cast<int>(sizeof(T))));
  if (slots < need_slots) return false;
  const int cpl = (panel / VEC + 31) / 32;
  const size_t smem = pipe_smem_bytes<T>();
  static bool attr_set[9] = {false};
  const int sms = num_sms();
  dim3 grid(static_cast<unsigned>(sms), static_cast<unsigned>((ncols + panel - 1) / panel));
#define FE_PIPE(CPL_)                                                                          \
  do {                                                                                         \
    auto kern = csr_spmm_pipe_kernel<T, VEC, CPL_>;                                            \
    if (!attr_set[CPL_]) {                                                                     \
      FE_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,    \
                                         static_cast<int>(smem)));                             \
      attr_set[CPL_] = true;                                                                   \
    }                                                                                          \
    kern<<<grid, kPipeWarps * 32, smem, s>>>(A.rows, A.rowptr, A.colind, vals, X, ldx, Y, ldy, \
                                             Z, ldz, ncols, panel, slots, alpha, gamma, beta,  \
                                             ug ? 1 : 0, ub ? 1 : 0, current_status_word());  \
    check_launch("csr_spmm_pipe_kernel");                                                      \
  } while (0)
  switch (cpl) {
    case 1: FE_PIPE(1); break;
    case 2: FE_PIPE(2); break;
    case 3: FE_PIPE(3); break;
    case 4: FE_PIPE(4); break;
    case 5: FE_PIPE(5); break;
    case 6: FE_PIPE(6); break;
    default: FE_PIPE(8); break;
  }
#undef FE_PIPE
  return true;
}

}  // namespace

int read_spmm_status(bool clear) {
  int v = 0;
  FE_CHECK_CUDA(cudaMemcpyFromSymbol(&v, g_spmm_status, sizeof(int)));
  if (clear && v != 0) {
    const int z = 0;
    FE_CHECK_CUDA(cudaMemcpyToSymbol(g_spmm_status, &z, sizeof(int)));
  }
  return v;
}

// Kernel selection for csr_spmm: "pipe" (bulk-copy pipelined) or "warp" (registers only).
// 0 = row-batched kernel (panels <= 96 vectors) where it applies, 1 = loop kernel,
// 2 = bulk-copy pipeline where it applies, 3 = row-batched with panels <= 64 vectors,
// 4 = mode 0 with the next Z row prefetched into L2.
static int g_spmm_mode = 0;
void set_spmm_mode(int mode) { g_spmm_mode = mode; }

template <typename T>
void fill_uniform(T* X, int64_t ld, int64_t n, int64_t m, uint64_t seed, cudaStream_t s);

// Kernel choice for a call: an explicit process-wide mode (1..3) wins; under the
// default mode a width tuned on this operator by fe_csr_autotune (within a factor
// of two of ncols) picks the kernel.
std::mutex g_tune_mutex;

int tuned_mode(const Csr& A, int precision, int64_t ncols) {
  if (g_spmm_mode != 0) return g_spmm_mode;
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  int best = -1;
  double best_d = 1.0;
  for (const auto& e : A.tuned[precision]) {
    if (e.mode < 0 || e.ncols <= 0) continue;
    const double d = std::fabs(std::log2(static_cast<double>(ncols) / e.ncols));
    if (d <= best_d) {
      best_d = d;
      best = e.mode;
    }
  }
  return best >= 0 ? best : 0;
}

template <typename T>
void csr_spmm_mode(int mode, const Csr& A, const T* X, int64_t ldx, T* Y, int64_t ldy, const T* Z,
                   int64_t ldz, int64_t ncols, double alpha, double gamma, double beta,
                   cudaStream_t s);

// Shared entry used by the C ABI and the host solver.
template <typename T>
void csr_spmm(const Csr& A, const T* X, int64_t ldx, T* Y, int64_t ldy, const T* Z, int64_t ldz,
              int64_t ncols, double alpha, double gamma, double beta, cudaStream_t s) {
  csr_spmm_mode<T>(tuned_mode(A, sizeof(T) == 4 ? 1 : 0, ncols), A, X, ldx, Y, ldy, Z, ldz, ncols,
                   alpha, gamma, beta, s);
}

template <typename T>
void csr_spmm_mode(int mode, const Csr& A, const T* X, int64_t ldx, T* Y, int64_t ldy, const T* Z,
                   int64_t ldz, int64_t ncols, double alpha, double gamma, double beta,
                   cudaStream_t s) {
  FE_REQUIRE(ncols >= 0 && ncols <= 0x7fffffff, "csr_spmm: invalid column count");
  if (ncols == 0 || A.rows == 0) return;
  FE_REQUIRE(X && Y, "csr_spmm: null block pointer");
  FE_REQUIRE(ldx >= ncols && ldy >= ncols, "csr_spmm: leading dimension smaller than ncols");
  const bool ub = beta != 0.0;
  const bool ug = gamma != 0.0;
  if (ub) {
    FE_REQUIRE(Z != nullptr && ldz >= ncols, "csr_spmm: beta != 0 needs a Z block");
  }
  FE_REQUIRE(!ranges_overlap(X, A.cols, ldx, ncols, static_cast<const T*>(Y), A.rows, ldy, ncols),
             "csr_spmm: X and Y overlap");
  const T* vals = nullptr;
  if constexpr (sizeof(T) == 8) vals = A.val64; else vals = A.val32;
  constexpr int VEC = VecT<T>::width;
  const bool vec_ok = ncols % VEC == 0 && ldx % VEC == 0 && ldy % VEC == 0 && aligned16(X) &&
                      aligned16(Y) && (!ub || (ldz % VEC == 0 && aligned16(Z)));
  if (vec_ok) {
    // Mode 0: the row-batched register kernel for slabs of >= 32 vectors and rows
    // of <= 8 nonzeros; mode 2: the bulk-copy pipelined kernel (needs 16-byte
    // aligned row gathers and rows that fit its stages).
    // Mode 0 gives each lane 8-byte vectors (up to 5 per lane, so a 320-column
    // FP32 slab needs no idle lanes and ~70 registers of loads in flight); mode 3
    // uses 16-byte vectors with at most 2 per lane.
    if (mode == 0 &&
        try_row_kernel<T, 8 / sizeof(T)>(A, vals, X, ldx, Y, ldy, Z, ldz, static_cast<int>(ncols),
                                         T(alpha), T(gamma), T(beta), ug, ub, s, 5))
      return;
    if (mode == 3 &&
        try_row_kernel<T, VEC>(A, vals, X, ldx, Y, ldy, Z, ldz, static_cast<int>(ncols), T(alpha),
                               T(gamma), T(beta), ug, ub, s, 2))
      return;
    // Mode 4: mode 0 with the next row's Z row prefetched into L2.
    if (mode == 4 &&
        try_row_kernel<T, 8 / sizeof(T)>(A, vals, X, ldx, Y, ldy, Z, ldz, static_cast<int>(ncols),
                                         T(alpha), T(gamma), T(beta), ug, ub, s, 5, true))
      return;
    // Mode 5: 16-byte vectors, up to 3 per lane (a 320-column FP32 slab in one panel);
    // mode 6: 8-byte vectors, up to 3 per lane (a 320-column FP32 slab in two panels,
    // fewer registers per warp).
    if (mode == 5 &&
        try_row_kernel<T, VEC>(A, vals, X, ldx, Y, ldy, Z, ldz, static_cast<int>(ncols), T(alpha),
                               T(gamma), T(beta), ug, ub, s, 3))
      return;
    if (mode == 6 &&
        try_row_kernel<T, 8 / sizeof(T)>(A, vals, X, ldx, Y, ldy, Z, ldz, static_cast<int>(ncols),
                                         T(alpha), T(gamma), T(beta), ug, ub, s, 3))
      return;
    // Mode 7: mode 0 with X and Z read through L2 only.
    if (mode == 7 &&
        try_row_kernel<T, 8 / sizeof(T)>(A, vals, X, ldx, Y, ldy, Z, ldz, static_cast<int>(ncols),
                                         T(alpha), T(gamma), T(beta), ug, ub, s, 5, false, true))
      return;
    if (mode == 2 && ncols * static_cast<int64_t>(sizeof(T)) >= 64 &&
        try_pipe<T, VEC>(A, vals, X, ldx, Y, ldy, Z, ldz, static_cast<int>(ncols), T(alpha),
                         T(gamma), T(beta), ug, ub, s))
      return;
  }
  // Where the selected kernel does not apply (too few 16-byte vectors for modes 3 and
  // 5, a block without 16-byte alignment or whole 16-byte rows), the row kernel with
  // 8-byte lanes runs before the loop kernels (mode 1 asks for the loop kernel).
  constexpr int V8 = 8 / sizeof(T);
  auto aligned8 = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 7u) == 0; };
  const bool vec8_ok = ncols % V8 == 0 && ldx % V8 == 0 && ldy % V8 == 0 && aligned8(X) &&
                       aligned8(Y) && (!ub || (ldz % V8 == 0 && aligned8(Z)));
  if (mode != 1 && vec8_ok &&
      try_row_kernel<T, V8>(A, vals, X, ldx, Y, ldy, Z, ldz, static_cast<int>(ncols), T(alpha),
                            T(gamma), T(beta), ug, ub, s, 5, false, mode == 7))
    return;
  if (vec_ok) {
    dispatch_vec<T, VEC>(A, vals, X, ldx, Y, ldy, Z, ldz, static_cast<int>(ncols), T(alpha),
                         T(gamma), T(beta), ug, ub, s);
  } else {
    dispatch_vec<T, 1>(A, vals, X, ldx, Y, ldy, Z, ldz, static_cast<int>(ncols), T(alpha),
                       T(gamma), T(beta), ug, ub, s);
  }
}

template void csr_spmm<double>(const Csr&, const double*, int64_t, double*, int64_t,
                               const double*, int64_t, int64_t, double, double, double,
                               cudaStream_t);

// Time every SpMM kernel on this operator for an n x ncols block in the Chebyshev
// step form (Y = a A X + g X + b Z, the filter's inner loop) and record the fastest
// in the operator's table. Returns the chosen mode.
template <typename T>
int autotune_spmm(Csr& A, int64_t ncols, cudaStream_t s) {
  FE_REQUIRE(ncols >= 1 && A.rows == A.cols, "autotune: invalid block width");
  const int64_t ld = ((ncols + 7) / 8) * 8;
  const size_t bytes = static_cast<size_t>(A.rows) * ld * sizeof(T);
  void *x = nullptr, *y = nullptr, *z = nullptr;
  FE_CHECK_CUDA(cudaMallocAsync(&x, bytes, s));
  FE_CHECK_CUDA(cudaMallocAsync(&y, bytes, s));
  FE_CHECK_CUDA(cudaMallocAsync(&z, bytes, s));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int best = 0;
  auto cleanup = [&] {
    cudaFreeAsync(x, s);
    cudaFreeAsync(y, s);
    cudaFreeAsync(z, s);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  };
  try {
    fill_uniform<T>(static_cast<T*>(x), ld, A.rows, ld, 11, s);
    fill_uniform<T>(static_cast<T*>(z), ld, A.rows, ld, 12, s);
    FE_CHECK_CUDA(cudaEventCreate(&e0));
    FE_CHECK_CUDA(cudaEventCreate(&e1));
    float best_ms = 0.0f;
    for (int mode : {0, 3, 2, 1, 4, 5, 6, 7}) {
      auto run = [&] {
        csr_spmm_mode<T>(mode, A, static_cast<const T*>(x), ld, static_cast<T*>(y), ld,
                         static_cast<const T*>(z), ld, ncols, 0.25, 0.1, -1.0, s);
      };
      run();  // warm-up (module load, caches)
      FE_CHECK_CUDA(cudaEventRecord(e0, s));
      for (int r = 0; r < 3; ++r) run();
      FE_CHECK_CUDA(cudaEventRecord(e1, s));
      FE_CHECK_CUDA(cudaEventSynchronize(e1));
      float ms = 0.0f;
      FE_CHECK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      if (mode == 0 || ms < best_ms) {
        best_ms = ms;
        best = mode;
      }
    }
  } catch (...) {
    cleanup();
    throw;
  }
  cleanup();
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  auto& table = A.tuned[sizeof(T) == 4 ? 1 : 0];
  int slot = -1;
  for (int i = 0; i < 4 && slot < 0; ++i)
    if (table[i].ncols == ncols || table[i].mode < 0) slot = i;
  if (slot < 0) {
    for (int i = 0; i < 3; ++i) table[i] = table[i + 1];
    slot = 3;
  }
  table[slot].ncols = static_cast<int32_t>(ncols);
  table[slot].mode = best;
  return best;
}
template int autotune_spmm<double>(Csr&, int64_t, cudaStream_t);
template int autotune_spmm<float>(Csr&, int64_t, cudaStream_t);
template void csr_spmm<float>(const Csr&, const float*, int64_t, float*, int64_t, const float*,
                              int64_t, int64_t, double, double, double, cudaStream_t);

// Y = alpha A X + gamma X + beta Z + R diag(delta) on FP32 blocks: the Chebyshev step
// of the refined filter's correction recurrence (see refined_filter in the solver).
// The row-batched kernel carries the extra term in its store; where that kernel does
// not apply, the step is followed by a separate column-scaled add.
void csr_spmm_corr_f32(const Csr& A, const float* X, int64_t ldx, float* Y, int64_t ldy,
                       const float* Z, int64_t ldz, const float* R, int64_t ldr,
                       const float* delta, int64_t ncols, double alpha, double gamma, double beta,
                       cudaStream_t s) {
  if (ncols == 0 || A.rows == 0) return;
  FE_REQUIRE(R && delta && ldr >= ncols, "csr_spmm_corr: invalid correction block");
  constexpr int VEC = 2;  // 8-byte lanes, as the default row kernel
  constexpr int NZ = 7;
  const bool ub = beta != 0.0;
  const int nvec = static_cast<int>(ncols / VEC);
  const bool ok = ncols % 4 == 0 && ldx % 4 == 0 && ldy % 4 == 0 && ldr % 4 == 0 &&
                  aligned16(X) && aligned16(Y) && aligned16(R) && aligned16(delta) &&
                  (!ub || (ldz % 4 == 0 && aligned16(Z))) && nvec >= 32 && A.max_row_nnz <= NZ &&
                  !ranges_overlap(X, A.cols, ldx, ncols, static_cast<const float*>(Y), A.rows,
                                  ldy, ncols);
  if (!ok) {
    csr_spmm<float>(A, X, ldx, Y, ldy, Z, ldz, ncols, alpha, gamma, beta, s);
    col_scaled_add_kernel<<<elementwise_grid(A.rows * ncols), 256, 0, s>>>(
        A.rows, static_cast<int>(ncols), R, ldr, delta, Y, ldy);
    check_launch("col_scaled_add_kernel");
    return;
  }
  const int max_cpl = 5;
  const int panels = (nvec + 32 * max_cpl - 1) / (32 * max_cpl);
  const int panel_vec = (nvec + panels - 1) / panels;
  const int cpl = (panel_vec + 31) / 32;
#define FE_ROWC(CPL_)                                                                          \
  do {                                                                                         \
    auto kern = csr_spmm_row_corr_kernel<float, VEC, CPL_, NZ>;                                \
    static int resident = 0;                                                                   \
    if (resident == 0) {                                                                       \
      FE_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, kern, kThreads,   \
                                                                  0));                         \
      resident = std::max(resident, 1);                                                        \
    }                                                                                          \
    int64_t blocks = std::min<int64_t>((A.rows + 7) / 8,                                       \
                                       static_cast<int64_t>(num_sms()) * resident);            \
    blocks = std::max<int64_t>(blocks, 1);                                                     \
    dim3 grid(static_cast<unsigned>(blocks), static_cast<unsigned>(panels));                   \
    kern<<<grid, kThreads, 0, s>>>(A.rows, A.rowptr, A.colind, A.val32, X, ldx, Y, ldy, Z, ldz, \
                                   static_cast<int>(ncols), panel_vec, static_cast<float>(alpha), \
                                   static_cast<float>(gamma), static_cast<float>(beta),        \
                                   gamma != 0.0 ? 1 : 0, ub ? 1 : 0, R, ldr, delta);           \
    check_launch("csr_spmm_row_corr_kernel");                                                  \
  } while (0)
  if (cpl == 1) FE_ROWC(1);
  else if (cpl == 2) FE_ROWC(2);
  else if (cpl == 3) FE_ROWC(3);
  else if (cpl == 4) FE_ROWC(4);
  else FE_ROWC(5);
#undef FE_ROWC
}

void refine_start(int64_t n, int64_t ncols, const double* R64, int64_t ld64, const double* X,
                  int64_t ldx, const double* theta, double c, float* R32, float* Z1,
                  int64_t ld32, cudaStream_t s) {
  if (n <= 0 || ncols <= 0) return;
  refine_start_kernel<<<elementwise_grid(n * ncols), 256, 0, s>>>(
      n, static_cast<int>(ncols), R64, ld64, X, ldx, theta, c, R32, Z1, ld32);
  check_launch("refine_start_kernel");
}

void refine_finish(int64_t n, int64_t ncols, const double* t, const float* Z, int64_t ld32,
                   double* X, int64_t ldx, cudaStream_t s) {
  if (n <= 0 || ncols <= 0) return;
  refine_finish_kernel<<<elementwise_grid(n * ncols), 256, 0, s>>>(
      n, static_cast<int>(ncols), t, Z, ld32, X, ldx);
  check_launch("refine_finish_kernel");
}

// In-place filter of degree `degree`: X <- T_degree(c*A + d*I) X, scratch holds Y_{k-1}.
// ---- multi-step filter host side ------------------------------------------
__global__ void csr_bandwidth_kernel(int64_t nrows, const int32_t* __restrict__ rowptr,
                                     const int32_t* __restrict__ colind,
                                     unsigned long long* __restrict__ out) {
  unsigned long long mx = 0;
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < nrows;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    for (int e = rowptr[r]; e < rowptr[r + 1]; ++e) {
      const int64_t dist = colind[e] >= r ? colind[e] - r : r - colind[e];
      mx = max(mx, static_cast<unsigned long long>(dist));
    }
  }
  for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0 && mx > 0) atomicMax(out, mx);
}

int64_t csr_bandwidth(const Csr& A, cudaStream_t s) {
  if (A.bandwidth >= 0) return A.bandwidth;
  unsigned long long* d = nullptr;
  FE_CHECK_CUDA(cudaMallocAsync(&d, sizeof(unsigned long long), s));
  FE_CHECK_CUDA(cudaMemsetAsync(d, 0, sizeof(unsigned long long), s));
  if (A.rows > 0) {
    csr_bandwidth_kernel<<<elementwise_grid(A.rows), 256, 0, s>>>(A.rows, A.rowptr, A.colind, d);
    check_launch("csr_bandwidth_kernel");
  }
  unsigned long long h = 0;
  FE_CHECK_CUDA(cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, s));
  FE_CHECK_CUDA(cudaFreeAsync(d, s));
  FE_CHECK_CUDA(cudaStreamSynchronize(s));
  A.bandwidth = static_cast<int64_t>(h);
  return A.bandwidth;
}

// 0 = off (default), 1 = on where it applies; 2..8 = that many steps per launch
// whatever the L2 window; 9 = one step per launch through the multi-step kernel;
// 12..18 = 2..8 steps per launch with plain (L1-cached) coherent loads; 100 P + S =
// P column panels (1, 2 or 4) of S steps per launch.
static int g_wave_mode = 0;
void set_wave_mode(int mode) { g_wave_mode = mode; }

size_t wave_sync_bytes(int64_t nrows) {
  const int64_t nblocks = ((std::max<int64_t>(nrows, 1) - 1) >> kWaveBlockShift) + 1;
  return 16 + sizeof(int) * static_cast<size_t>(kWaveMaxLevels) * nblocks;
}

template <typename T, int VEC, int CPL, int LOADS>
void launch_wave_coop(dim3 g, const WaveParams<T>& P, cudaStream_t s) {
  WaveParams<T> arg = P;
  void* args[] = {&arg};
  FE_CHECK_CUDA(cudaLaunchCooperativeKernel(
      reinterpret_cast<const void*>(cheb_wave_kernel<T, VEC, CPL, 7, LOADS>), g, dim3(kThreads),
      args, 0, s));
}

template <typename T, int VEC, int LOADS>
void launch_wave(int cpl, dim3 g, const WaveParams<T>& P, cudaStream_t s) {
  switch (cpl) {
    case 1: launch_wave_coop<T, VEC, 1, LOADS>(g, P, s); break;
    case 2: launch_wave_coop<T, VEC, 2, LOADS>(g, P, s); break;
    case 3: launch_wave_coop<T, VEC, 3, LOADS>(g, P, s); break;
    case 4: launch_wave_coop<T, VEC, 4, LOADS>(g, P, s); break;
    default: launch_wave_coop<T, VEC, 5, LOADS>(g, P, s); break;
  }
}

template <typename T, int CPL>
int wave_resident() {
  static int resident = 0;  // per instantiation; the same on every B200
  if (resident == 0) {
    FE_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &resident, cheb_wave_kernel<T, 8 / sizeof(T), CPL, 7, 1>, kThreads, 0));
    resident = std::max(resident, 1);
  }
  return resident;
}

template <typename T>
int wave_resident_for(int cpl) {
  switch (cpl) {
    case 1: return wave_resident<T, 1>();
    case 2: return wave_resident<T, 2>();
    case 3: return wave_resident<T, 3>();
    case 4: return wave_resident<T, 4>();
    default: return wave_resident<T, 5>();
  }
}

// The filter Y_degree = T_degree(c A + d I) X (X and Sc as in cheb_filter; the result
// lands in X) in launches of several steps each, over column panels where a panel's
// window of 2 bw rows per level must fit in L2. Returns false, having launched
// nothing, where the multi-step kernel does not apply (not square, rows longer than
// 7, blocks not made of 8-byte vectors, or no panel split whose window fits about
// 75% of L2 with at least two levels); the caller then runs one step per launch.
template <typename T>
bool cheb_filter_wave(const Csr& A, T* X, int64_t ldx, T* Sc, int64_t lds, int64_t ncols,
                      int degree, double c, double d, void* sync, size_t sync_bytes,
                      cudaStream_t s) {
  constexpr int VEC = 8 / sizeof(T);
  const int mode = g_wave_mode;
  if (mode == 0 || degree < 2 || A.rows != A.cols || A.rows < 4096 || A.max_row_nnz > 7 ||
      A.max_row_nnz < 1)
    return false;
  if (!sync || sync_bytes < wave_sync_bytes(A.rows)) return false;
  if (ncols % VEC != 0 || ldx % VEC != 0 || lds % VEC != 0 || !aligned16(X) || !aligned16(Sc))
    return false;
  if (ranges_overlap(X, A.rows, ldx, ncols, static_cast<const T*>(Sc), A.rows, lds, ncols))
    return false;
  const int64_t bw = csr_bandwidth(A, s);
  int dev = 0, l2 = 0;
  FE_CHECK_CUDA(cudaGetDevice(&dev));
  FE_CHECK_CUDA(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev));
  const double budget = 0.75 * static_cast<double>(l2);
  // Candidate splits: P panels of ncols / P columns (16-byte aligned panel starts,
  // 32..160 vectors each); S levels with (S + 1) windows of 2 bw rows in L2. Cost per
  // step in bytes: the CSR once per panel plus (2 + S) / S passes over the blocks.
  int panels = 0, levels = 0, loads = 1;
  double best = 0.0;
  const double csr_bytes = static_cast<double>(A.nnz) * (4.0 + sizeof(T));
  const double block_bytes = static_cast<double>(A.rows) * ncols * sizeof(T);
  const int force_p = mode >= 100 ? mode / 100 : 0;
  for (int P : {1, 2, 4}) {
    if (ncols % P != 0 || (force_p && P != force_p)) continue;
    const int64_t pc = ncols / P;
    const int64_t pv = pc / VEC;
    if (pc % VEC != 0 || pv < 32 || pv > 160 || (P > 1 && (pc * sizeof(T)) % 16 != 0)) continue;
    const double window = 2.0 * static_cast<double>(bw) * pc * sizeof(T);
    int S = 0;
    if (mode >= 100) S = std::min(mode % 100, degree);
    else if (mode >= 2 && mode <= 8) S = std::min(mode, degree);
    else if (mode >= 12 && mode <= 18) S = std::min(mode - 10, degree);
    else if (mode == 9) S = 1;
    else
      for (int t = std::min(kWaveMaxLevels, degree); t >= 2 && S == 0; --t)
        if ((t + 1) * window <= budget) S = t;
    if (S == 0) continue;
    const double cost = P * csr_bytes + block_bytes * (2.0 + S) / S;
    if (panels == 0 || cost < best) {
      best = cost;
      panels = P;
      levels = S;
    }
    if (mode >= 2) break;  // forced schedules take the fewest panels that fit
  }
  if (panels == 0 || levels < 1) return false;
  if (mode >= 12 && mode <= 18) loads = 2;
  if (mode == 9) loads = 3;
  const int64_t pc = ncols / panels;
  const int64_t pv = pc / VEC;
  const int cpl = static_cast<int>((pv + 31) / 32);
  const int64_t grid = static_cast<int64_t>(num_sms()) * wave_resident_for<T>(cpl);
  const int64_t nblocks = ((A.rows - 1) >> kWaveBlockShift) + 1;
  int* status = current_status_word();
  char* base = static_cast<char*>(sync);
  for (int p = 0; p < panels; ++p) {
    for (int k0 = 1; k0 <= degree; k0 += levels) {
      const int lv = std::min(levels, degree - k0 + 1);
      WaveParams<T> P{};
      P.nrows = A.rows;
      P.rowptr = A.rowptr;
      P.colind = A.colind;
      if constexpr (sizeof(T) == 8) P.vals = A.val64; else P.vals = A.val32;
      P.buf[0] = X + p * pc;
      P.buf[1] = Sc + p * pc;
      P.ld[0] = ldx;
      P.ld[1] = lds;
      P.ncols = static_cast<int>(pc);
      P.panel_vec = static_cast<int>(pv);
      P.levels = lv;
      P.first_k = k0;
      for (int l = 0; l < lv; ++l) {
        const bool first = k0 + l == 1;
        P.alpha[l] = static_cast<T>(first ? c : 2.0 * c);
        P.gamma[l] = static_cast<T>(first ? d : 2.0 * d);
        P.beta[l] = static_cast<T>(first ? 0.0 : -1.0);
      }
      P.reach = bw;
      P.abort_flag = reinterpret_cast<int*>(base);
      P.done = reinterpret_cast<int*>(base + 16);
      P.nblocks = nblocks;
      P.status = status;
      P.max_polls = 1LL << 22;
      FE_CHECK_CUDA(cudaMemsetAsync(sync, 0, 16 + sizeof(int) * lv * nblocks, s));
      const dim3 g(static_cast<unsigned>(grid), 1);
      if (loads == 1) launch_wave<T, VEC, 1>(cpl, g, P, s);
      else if (loads == 2) launch_wave<T, VEC, 2>(cpl, g, P, s);
      else launch_wave<T, VEC, 3>(cpl, g, P, s);
      check_launch("cheb_wave_kernel");
    }
  }
  if (degree % 2 == 1) {  // Y_degree is in buf[1]
    FE_CHECK_CUDA(cudaMemcpy2DAsync(X, ldx * sizeof(T), Sc, lds * sizeof(T), ncols * sizeof(T),
                                    A.rows, cudaMemcpyDeviceToDevice, s));
  }
  return true;
}

template bool cheb_filter_wave<float>(const Csr&, float*, int64_t, float*, int64_t, int64_t, int,
                                      double, double, void*, size_t, cudaStream_t);
template bool cheb_filter_wave<double>(const Csr&, double*, int64_t, double*, int64_t, int64_t,
                                       int, double, double, void*, size_t, cudaStream_t);

template <typename T>
void cheb_filter(const Csr& A, T* X, T* scratch, int64_t ld, int64_t ncols, int degree, double c,
                 double d, cudaStream_t s) {
  FE_REQUIRE(degree >= 1, "cheb_filter: degree must be >= 1");
  if (degree >= 2 && g_wave_mode != 0 && A.rows == A.cols) {
    // several steps per launch where the operator's bandwidth allows it
    const size_t bytes = wave_sync_bytes(A.rows);
    void* sync = nullptr;
    FE_CHECK_CUDA(cudaMallocAsync(&sync, bytes, s));
    bool done = false;
    try {
      done = cheb_filter_wave<T>(A, X, ld, scratch, ld, ncols, degree, c, d, sync, bytes, s);
    } catch (...) {
      cudaFreeAsync(sync, s);
      throw;
    }
    FE_CHECK_CUDA(cudaFreeAsync(sync, s));
    if (done) return;
  }
  // Y1 = c*A*Y0 + d*Y0 into scratch; then Y_k overwrites Y_{k-2} in place.
  csr_spmm<T>(A, X, ld, scratch, ld, nullptr, 0, ncols, c, d, 0.0, s);
  T* prev = X;       // Y_{k-2}
  T* cur = scratch;  // Y_{k-1}
  for (int k = 2; k <= degree; ++k) {
    csr_spmm<T>(A, cur, ld, prev, ld, prev, ld, ncols, 2.0 * c, 2.0 * d, -1.0, s);
    std::swap(prev, cur);
  }
  if (cur != X) {
    FE_CHECK_CUDA(cudaMemcpy2DAsync(X, ld * sizeof(T), cur, ld * sizeof(T), ncols * sizeof(T),
                                    A.rows, cudaMemcpyDeviceToDevice, s));
  }
}

template void cheb_filter<double>(const Csr&, double*, double*, int64_t, int64_t, int, double,
                                  double, cudaStream_t);
template void cheb_filter<float>(const Csr&, float*, float*, int64_t, int64_t, int, double,
                                 double, cudaStream_t);

}  // namespace fe

using fe::guarded;

extern "C" int fe_spmm_csr_f64(fe_csr_t A, const double* X, int64_t ldx, double* Y, int64_t ldy,
                               int64_t ncols, double alpha, double beta, void* stream) {
  return guarded("fe_spmm_csr_f64", [&] {
    FE_REQUIRE(A, "null CSR handle");
    fe::csr_spmm<double>(A->m, X, ldx, Y, ldy, Y, ldy, ncols, alpha, 0.0, beta,
                         fe::as_stream(stream));
  });
}

extern "C" int fe_spmm_csr_f32(fe_csr_t A, const float* X, int64_t ldx, float* Y, int64_t ldy,
                               int64_t ncols, double alpha, double beta, void* stream) {
  return guarded("fe_spmm_csr_f32", [&] {
    FE_REQUIRE(A, "null CSR handle");
    fe::csr_spmm<float>(A->m, X, ldx, Y, ldy, Y, ldy, ncols, alpha, 0.0, beta,
                        fe::as_stream(stream));
  });
}

extern "C" int fe_cheb_step_f64(fe_csr_t A, const double* Ycur, const double* Yprev,
                                double* Yout, int64_t ld, int64_t ncols, double alpha,
                                double gamma, double beta, void* stream) {
  return guarded("fe_cheb_step_f64", [&] {
    FE_REQUIRE(A, "null CSR handle");
    fe::csr_spmm<double>(A->m, Ycur, ld, Yout, ld, Yprev, ld, ncols, alpha, gamma, beta,
                         fe::as_stream(stream));
  });
}

extern "C" int fe_cheb_step_f32(fe_csr_t A, const float* Ycur, const float* Yprev, float* Yout,
                                int64_t ld, int64_t ncols, double alpha, double gamma,
                                double beta, void* stream) {
  return guarded("fe_cheb_step_f32", [&] {
    FE_REQUIRE(A, "null CSR handle");
    fe::csr_spmm<float>(A->m, Ycur, ld, Yout, ld, Yprev, ld, ncols, alpha, gamma, beta,
                        fe::as_stream(stream));
  });
}

extern "C" int fe_cheb_filter_f64(fe_csr_t A, double* X, double* scratch, int64_t ld,
                                  int64_t ncols, int32_t degree, double c, double d,
                                  void* stream) {
  return guarded("fe_cheb_filter_f64", [&] {
    FE_REQUIRE(A, "null CSR handle");
    fe::cheb_filter<double>(A->m, X, scratch, ld, ncols, degree, c, d, fe::as_stream(stream));
  });
}

extern "C" int fe_cheb_filter_f32(fe_csr_t A, float* X, float* scratch, int64_t ld,
                                  int64_t ncols, int32_t degree, double c, double d,
                                  void* stream) {
  return guarded("fe_cheb_filter_f32", [&] {
    FE_REQUIRE(A, "null CSR handle");
    fe::cheb_filter<float>(A->m, X, scratch, ld, ncols, degree, c, d, fe::as_stream(stream));
  });
}

extern "C" int fe_csr_autotune(fe_csr_t A, int64_t ncols, int32_t precision, void* stream,
                               int32_t* mode) {
  return fe::guarded("fe_csr_autotune", [&] {
    FE_REQUIRE(A, "null CSR handle");
    FE_REQUIRE(precision == 0 || precision == 1, "precision must be 0 (FP64) or 1 (FP32)");
    FE_CHECK_CUDA(cudaSetDevice(A->m.device));
    const int m = precision == 0 ? fe::autotune_spmm<double>(A->m, ncols, fe::as_stream(stream))
                                 : fe::autotune_spmm<float>(A->m, ncols, fe::as_stream(stream));
    if (mode) *mode = m;
  });
}
