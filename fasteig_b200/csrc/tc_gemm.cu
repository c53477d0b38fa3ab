// Tensor-core (tcgen05, TMEM accumulators, TMA-fed) split-TF32 kernels for the
// tall-skinny FP32 block products of the mixed-precision path:
//
//   Gram      G = X^T Y           (X: n x k, Y: n x m; reduction over the n rows)
//   Rotation  Y = alpha X C + beta Y  (X: n x k, C: k x m FP64 column-major)
//
// They replace the reference's cublasDgemm calls in transpose_multiply
// (src/gpu/CudaMultiVector.cpp:395-405), right_multiply_active_columns (:353-358)
// and Cholesky QR (src/core/Orthogonalization.cpp:202-235) for FP32 blocks.
//
// Precision ("3xTF32"): every FP32 operand x is split into x_hi = rna_tf32(x) and
// x_lo = rna_tf32(x - x_hi), and the product is accumulated in FP32 TMEM as
// x_hi*y_hi + x_hi*y_lo + x_lo*y_hi. Products of TF32 values are exact in FP32 and
// the dropped x_lo*y_lo term is below 2^-22 |x y|, so the result carries FP32-level
// error. The Gram is split over row chunks whose FP32 partial tiles are summed in
// FP64 in a fixed order (deterministic).
//
// Pipeline per CTA (128-row MMA tile, N-tile of 160 columns, 3 smem stages):
//   warp 0 lane 0 : TMA producer (2D tiled loads, 128-byte swizzle)
//   warp 1        : TMEM allocator; lane 0 issues tcgen05.mma and commits
//   warps 2..5    : split FP32 tiles into hi/lo in shared memory, then drain
//                   TMEM (tcgen05.ld 32x32b) in the epilogue
// All mbarrier waits are bounded; on timeout the kernel records an error code in
// a device status word (fe_device_status) and leaves.

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>

#include "fe_common.cuh"

namespace fe {

int read_spmm_status(bool clear);
void set_spmm_mode(int mode);
void set_wave_mode(int mode);
void set_f64_gemm_mode(int mode);

__device__ int g_tc_status = 0;  // 0 = ok, otherwise a code of the first failed wait

// Aligned 3xTF32 rotations on the persistent kernel (1) or one CTA per tile (0).
static int g_rotate_persistent = 2;  // 2: TMEM A operand, 1: shared-memory split, 0: per tile
void set_rotate_persistent(int on) { g_rotate_persistent = on; }

namespace {

constexpr int kM = 128;           // MMA M (TMEM lanes)
constexpr int kN = 160;           // MMA N (columns per CTA tile)
constexpr int kKB = 32;           // FP32 elements per 128-byte swizzle row
constexpr int kStages = 3;
constexpr int kThreads = 192;     // 6 warps
// The Gram splits both operands (36 KB per K stage against the rotation's 16 KB),
// so it runs 8 splitting warps.
constexpr int kGramSplitThreads = 256;
constexpr int kGramThreads = 64 + kGramSplitThreads;
constexpr int kSplitThreads = 128;
constexpr uint32_t kTmemCols = 256;

// Per-stage shared memory (bytes); every buffer is 1024-byte aligned.
constexpr int kABytes = kM * kKB * 4;   // 16 KB
constexpr int kBBytes = kN * kKB * 4;   // 20 KB
constexpr int kStageBytes = 2 * kABytes + 2 * kBBytes;
constexpr int kSmemBytes = kStages * kStageBytes + 1024 /*align*/ + 256 /*barriers*/;
// Rotation epilogue staging: 4 warps x 32 rows x (kN + 1) floats inside the stages.
constexpr int kStageLd = kN + 1;
static_assert(4 * 32 * kStageLd * 4 <= kStages * kStageBytes, "epilogue staging does not fit");

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Non-blocking test of a phase (try_wait may suspend the thread for a while first).
__device__ __forceinline__ bool mbar_test_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: `limit` SM clocks (about two seconds by default), then record `code`
// in the launch's status word and give up.
__device__ __forceinline__ bool mbar_wait_limit(uint64_t* bar, uint32_t parity, int code,
                                                int* status, long long limit) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (true) {
    for (int i = 0; i < 64; ++i)
      if (mbar_try_wait(bar, parity)) return true;
    if (clock64() - t0 > limit) {
      atomicCAS(status, 0, code);
      return false;
    }
  }
}

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int code, int* status) {
  return mbar_wait_limit(bar, parity, code, status, 4000000000LL);
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// UMMA shared-memory descriptor (SM100 version 1). Layout types: 2 = 128-byte
// swizzle of 16-byte chunks (K-major operands); 1 = 128-byte swizzle of 32-byte
// chunks, the only MN-major layout the tensor cores accept for TF32.
constexpr uint32_t kLayoutSW128 = 2;
constexpr uint32_t kLayoutSW128Base32 = 1;

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo_bytes,
                                              uint32_t sbo_bytes, uint32_t layout) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((addr >> 4) & 0x3FFFu);
  d |= static_cast<uint64_t>((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= static_cast<uint64_t>((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= static_cast<uint64_t>(1) << 46;  // version (SM100)
  d |= static_cast<uint64_t>(layout & 7u) << 61;
  return d;
}

// Instruction descriptor: kind::tf32, FP32 accumulate, M = 128, N = kN.
__host__ __device__ constexpr uint32_t idesc_tf32(bool a_mn_major, bool b_mn_major) {
  return (1u << 4)                               // c_format = F32
         | (2u << 7)                             // a_format = TF32
         | (2u << 10)                            // b_format = TF32
         | (static_cast<uint32_t>(a_mn_major) << 15) |
         (static_cast<uint32_t>(b_mn_major) << 16) |
         (static_cast<uint32_t>(kN >> 3) << 17)  // n_dim
         | (static_cast<uint32_t>(kM >> 4) << 24);  // m_dim
}

__device__ __forceinline__ void umma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// The same MMA with A read from tensor memory (row i of A in TMEM lane i, one FP32/TF32
// element per 32-bit column, K consecutive columns), B from shared memory.
__device__ __forceinline__ void umma_tf32_ta(uint32_t d_tmem, uint32_t a_tmem, uint64_t bdesc,
                                             uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d_tmem),
      "r"(a_tmem), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const float* v) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15, %16};" ::"r"(taddr),
      "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
      "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
      "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])), "r"(__float_as_uint(v[8])),
      "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
      "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])),
      "r"(__float_as_uint(v[15]))
      : "memory");
}

__device__ __forceinline__ uint32_t tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void split4(const float4& v, float4& hi, float4& lw) {
  hi.x = __uint_as_float(tf32_rna(v.x));
  hi.y = __uint_as_float(tf32_rna(v.y));
  hi.z = __uint_as_float(tf32_rna(v.z));
  hi.w = __uint_as_float(tf32_rna(v.w));
  lw.x = __uint_as_float(tf32_rna(v.x - hi.x));
  lw.y = __uint_as_float(tf32_rna(v.y - hi.y));
  lw.z = __uint_as_float(tf32_rna(v.z - hi.z));
  lw.w = __uint_as_float(tf32_rna(v.w - hi.w));
}

// Split n_vec16 16-byte chunks of raw FP32 data in place into hi, and into lo
// (NT splitting threads, this one `tid`).
template <int NT = kSplitThreads>
__device__ __forceinline__ void split_tile(float* raw_hi, float* lo, int n_vec16, int tid) {
  float4* h = reinterpret_cast<float4*>(raw_hi);
  float4* l = reinterpret_cast<float4*>(lo);
  for (int i = tid; i < n_vec16; i += NT) {
    float4 hi, lw;
    split4(h[i], hi, lw);
    h[i] = hi;
    l[i] = lw;
  }
}

// As split_tile, for the last K stage of a Gram row chunk: the data are TMA boxes
// of 32 rows of 128 bytes (the 128-byte swizzle permutes 16-byte chunks within a
// row only), and rows whose index within their box is >= `valid` lie past the
// chunk's end; they are written as zeros so they do not enter this chunk's sum.
template <int NT = kSplitThreads>
__device__ __forceinline__ void split_tile_rows(float* raw_hi, float* lo, int n_vec16, int tid,
                                                int valid) {
  float4* h = reinterpret_cast<float4*>(raw_hi);
  float4* l = reinterpret_cast<float4*>(lo);
  for (int i = tid; i < n_vec16; i += NT) {
    float4 hi = make_float4(0.f, 0.f, 0.f, 0.f), lw = hi;
    if (((i >> 3) & 31) < valid) split4(h[i], hi, lw);
    h[i] = hi;
    l[i] = lw;
  }
}

struct Smem {
  uint8_t* base;  // 1024-aligned
  uint64_t* full;
  uint64_t* empty;
  uint64_t* split;
  uint64_t* accum;
  uint32_t* tmem_slot;
  uint64_t* sub_full;   // Gram: a sub-chunk accumulator is complete (2, by buffer)
  uint64_t* sub_empty;  // Gram: a sub-chunk accumulator has been drained (2)
  int* status;  // the launch's status word (a solve's own, or the library default)
  __device__ float* a_hi(int s) const { return reinterpret_cast<float*>(base + s * kStageBytes); }
  __device__ float* a_lo(int s) const {
    return reinterpret_cast<float*>(base + s * kStageBytes + kABytes);
  }
  __device__ float* b_hi(int s) const {
    return reinterpret_cast<float*>(base + s * kStageBytes + 2 * kABytes);
  }
  __device__ float* b_lo(int s) const {
    return reinterpret_cast<float*>(base + s * kStageBytes + 2 * kABytes + kBBytes);
  }
};

__device__ __forceinline__ Smem carve(uint8_t* dyn, int* status) {
  Smem s;
  s.status = status ? status : &g_tc_status;
  uintptr_t p = reinterpret_cast<uintptr_t>(dyn);
  p = (p + 1023) & ~uintptr_t(1023);
  s.base = reinterpret_cast<uint8_t*>(p);
  uint64_t* bars = reinterpret_cast<uint64_t*>(s.base + kStages * kStageBytes);
  s.full = bars;
  s.empty = bars + kStages;
  s.split = bars + 2 * kStages;
  s.accum = bars + 3 * kStages;
  s.tmem_slot = reinterpret_cast<uint32_t*>(bars + 3 * kStages + 1);
  s.sub_full = bars + 3 * kStages + 2;
  s.sub_empty = bars + 3 * kStages + 4;
  return s;
}

// Common prologue: barrier init (thread 0) and TMEM allocation (warp 1).
__device__ __forceinline__ void prologue(const Smem& sm, int warp,
                                         int split_warps = kSplitThreads / 32,
                                         uint32_t tmem_cols = kTmemCols) {
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&sm.full[s], 1);
      mbar_init(&sm.empty[s], 1);
      mbar_init(&sm.split[s], split_warps);
    }
    mbar_init(sm.accum, 1);
    for (int b = 0; b < 2; ++b) {
      mbar_init(&sm.sub_full[b], 1);
      mbar_init(&sm.sub_empty[b], split_warps);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    fence_proxy_async();
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(sm.tmem_slot)),
                 "r"(tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
}

__device__ __forceinline__ void epilogue_dealloc(const Smem& sm, int warp, uint32_t tmem,
                                                 uint32_t tmem_cols = kTmemCols) {
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(tmem_cols)
                 : "memory");
  }
}

// MMA issue loop shared by both kernels. Operand descriptors per K-step (8
// elements of K): K-major tiles advance 32 bytes inside the 128-byte swizzle
// row; MN-major tiles advance 8 rows (1024 bytes, two 4-row swizzle atoms).
template <bool kMN>
__device__ void mma_loop(const Smem& sm, uint32_t tmem, int nkb, uint32_t idesc) {
  // K-major (16-byte swizzle atoms of 8 rows x 128 B): SBO = 1024, LBO unused (16).
  // MN-major (32-byte swizzle atoms of 4 rows x 128 B): LBO = bytes between
  // 32-element column groups (one TMA box of 32 rows x 128 B = 4096), SBO = 512
  // between 4-row groups.
  const uint32_t lbo = kMN ? 4096u : 16u;
  const uint32_t sbo = kMN ? 512u : 1024u;
  const uint32_t layout = kMN ? kLayoutSW128Base32 : kLayoutSW128;
  for (int kb = 0; kb < nkb; ++kb) {
    const int s = kb % kStages;
    const uint32_t ph = (kb / kStages) & 1u;
    if (!mbar_wait(&sm.split[s], ph, 3, sm.status)) return;
    tc_fence_after();
    const uint32_t ah = smem_u32(sm.a_hi(s)), al = smem_u32(sm.a_lo(s));
    const uint32_t bh = smem_u32(sm.b_hi(s)), bl = smem_u32(sm.b_lo(s));
#pragma unroll
    for (int k = 0; k < kKB / 8; ++k) {
      const uint32_t off = kMN ? k * 1024u : k * 32u;
      const uint64_t dah = smem_desc(ah + off, lbo, sbo, layout);
      const uint64_t dal = smem_desc(al + off, lbo, sbo, layout);
      const uint64_t dbh = smem_desc(bh + off, lbo, sbo, layout);
      const uint64_t dbl = smem_desc(bl + off, lbo, sbo, layout);
      const uint32_t acc = (kb > 0 || k > 0) ? 1u : 0u;
      umma_tf32(tmem, dah, dbh, idesc, acc);
      umma_tf32(tmem, dah, dbl, idesc, 1u);
      umma_tf32(tmem, dal, dbh, idesc, 1u);
    }
    umma_commit(&sm.empty[s]);
  }
  umma_commit(sm.accum);
}

// Gram MMA loop: the row chunk runs as sub-chunks of kGramSubStages K stages, each
// accumulated from zero into one of two TMEM buffers (columns 0 and 256, alternating);
// sub_full[b] fires when a sub-chunk's products are complete, and buffer b is reused
// only after the split warps have drained it (sub_empty[b]).
constexpr int kGramSubStages = 8;  // 256 rows
constexpr uint32_t kGramTmemCols = 512;

__device__ void mma_loop_gram(const Smem& sm, uint32_t tmem, int nkb, uint32_t idesc) {
  const uint32_t lbo = 4096u, sbo = 512u, layout = kLayoutSW128Base32;  // MN-major operands
  for (int kb = 0; kb < nkb; ++kb) {
    const int s = kb % kStages;
    const uint32_t ph = (kb / kStages) & 1u;
    const int sub = kb / kGramSubStages;
    const int buf = sub & 1;
    const bool first = kb % kGramSubStages == 0;
    if (first && sub >= 2) {
      if (!mbar_wait(&sm.sub_empty[buf], static_cast<uint32_t>((sub >> 1) - 1) & 1u, 5,
                     sm.status))
        return;
      tc_fence_after();
    }
    if (!mbar_wait(&sm.split[s], ph, 3, sm.status)) return;
    tc_fence_after();
    const uint32_t d = tmem + static_cast<uint32_t>(buf) * 256u;
    const uint32_t ah = smem_u32(sm.a_hi(s)), al = smem_u32(sm.a_lo(s));
    const uint32_t bh = smem_u32(sm.b_hi(s)), bl = smem_u32(sm.b_lo(s));
#pragma unroll
    for (int k = 0; k < kKB / 8; ++k) {
      const uint32_t off = k * 1024u;
      const uint64_t dah = smem_desc(ah + off, lbo, sbo, layout);
      const uint64_t dal = smem_desc(al + off, lbo, sbo, layout);
      const uint64_t dbh = smem_desc(bh + off, lbo, sbo, layout);
      const uint64_t dbl = smem_desc(bl + off, lbo, sbo, layout);
      const uint32_t acc = (!first || k > 0) ? 1u : 0u;
      umma_tf32(d, dah, dbh, idesc, acc);
      umma_tf32(d, dah, dbl, idesc, 1u);
      umma_tf32(d, dal, dbh, idesc, 1u);
    }
    umma_commit(&sm.empty[s]);
    if ((kb + 1) % kGramSubStages == 0 || kb + 1 == nkb) umma_commit(&sm.sub_full[buf]);
  }
}

// ------------------------------------------------------------------ Gram ----
// grid.x = k_tiles * m_tiles (k tile fastest), grid.y = row chunks.
// A = X^T (MN-major: 4 boxes of 32 columns x 32 rows), B = Y (MN-major, 5 boxes).
// X and Y tensor maps start at columns aligned down to 16 bytes; sx/sy are the
// column shifts of the caller's views (outputs are re-indexed). Warps: 0 TMA
// producer, 1 MMA issuer, 2-9 hi/lo split, then epilogue.
__global__ void __launch_bounds__(kGramThreads, 1)
gram_tc_kernel(const __grid_constant__ CUtensorMap tmX, const __grid_constant__ CUtensorMap tmY,
               int64_t n, int k, int m, int sx, int sy, int k_tiles, int64_t rows_per_chunk,
               float* __restrict__ partial, int symmetric, int* status) {
  extern __shared__ uint8_t dyn_smem[];
  const Smem sm = carve(dyn_smem, status);
  const int warp = threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  const int ti = blockIdx.x % k_tiles;
  const int tj = blockIdx.x / k_tiles;
  const int i0 = ti * kM;   // tile origin in shifted (tensor-map) column space of X
  const int j0 = tj * kN;
  // X^T X: a tile wholly below the diagonal is the transpose of a computed one.
  if (symmetric && i0 >= j0 + kN) return;
  const int64_t r_begin = static_cast<int64_t>(blockIdx.y) * rows_per_chunk;
  const int64_t r_end = min(n, r_begin + rows_per_chunk);
  const int nkb = static_cast<int>((r_end - r_begin + kKB - 1) / kKB);

  prologue(sm, warp, kGramSplitThreads / 32, kGramTmemCols);
  const uint32_t tmem = *sm.tmem_slot;

  if (warp == 0 && lane == 0) {
    for (int kb = 0; kb < nkb; ++kb) {
      const int s = kb % kStages;
      const uint32_t ph = (kb / kStages) & 1u;
      if (!mbar_wait(&sm.empty[s], ph ^ 1u, 1, sm.status)) break;
      mbar_expect_tx(&sm.full[s], kABytes + kBBytes);
      const int y = static_cast<int>(r_begin + static_cast<int64_t>(kb) * kKB);
#pragma unroll
      for (int c = 0; c < kM / 32; ++c)
        tma_load_2d(sm.a_hi(s) + c * (32 * kKB), &tmX, i0 + 32 * c, y, &sm.full[s]);
#pragma unroll
      for (int c = 0; c < kN / 32; ++c)
        tma_load_2d(sm.b_hi(s) + c * (32 * kKB), &tmY, j0 + 32 * c, y, &sm.full[s]);
    }
  } else if (warp == 1) {
    if (lane == 0) mma_loop_gram(sm, tmem, nkb, idesc_tf32(true, true));
    __syncwarp();
  } else if (warp >= 2) {
    const int tid = threadIdx.x - 64;
    // TMEM: the MMA's sub-chunk buffers at columns [0, kN) and [256, 256 + kN); the
    // running sum at [160, 240) and [416, 496) (this warp's half of the columns).
    // Each split warp owns TMEM lanes 32 (warp % 4) .. + 31 and half of the columns,
    // and drains completed sub-chunks into the running sum in FP32 registers
    // (round to nearest): the tensor-core accumulator's own rounding error then
    // grows with the 256 rows of a sub-chunk instead of the whole chunk.
    const int q = warp % 4;
    const int c0 = ((warp - 2) / 4) * (kN / 2);
    const uint32_t lane_base = tmem + (static_cast<uint32_t>(q * 32) << 16);
    auto t2col = [](int c) -> uint32_t {
      return c < kN / 2 ? 160u + static_cast<uint32_t>(c) : 336u + static_cast<uint32_t>(c);
    };
    const int nsub = (nkb + kGramSubStages - 1) / kGramSubStages;
    int drained = 0;
    bool failed = false;
    auto drain = [&](int j) {
      const uint32_t src = lane_base + static_cast<uint32_t>(j & 1) * 256u;
      for (int c = c0; c < c0 + kN / 2; c += 16) {
        float v[16];
        tmem_ld16(src + c, v);
        if (j > 0) {
          float t[16];
          tmem_ld16(lane_base + t2col(c), t);
#pragma unroll
          for (int e = 0; e < 16; ++e) v[e] += t[e];
        }
        tmem_st16(lane_base + t2col(c), v);
      }
      asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&sm.sub_empty[j & 1]);
    };
    // Drain the next sub-chunk if its products are complete (decided for the whole
    // warp: tcgen05 loads and stores are warp-collective).
    auto try_drain = [&]() {
      if (drained >= nsub) return;
      // every lane observes the phase (acquire) before the warp reads TMEM
      if (__all_sync(0xffffffffu,
                     mbar_test_wait(&sm.sub_full[drained & 1], (drained >> 1) & 1))) {
        tc_fence_after();
        drain(drained);
        ++drained;
      }
    };
    // Rows past r_end inside the last block belong to the next chunk: the split
    // writes them as zeros, so they do not enter this chunk's sum.
    for (int kb = 0; kb < nkb && !failed; ++kb) {
      const int s = kb % kStages;
      const uint32_t ph = (kb / kStages) & 1u;
      // wait for the stage's operands, draining finished sub-chunks meanwhile (the
      // MMA may be waiting for a drain before it frees this stage's buffers)
      const long long t0 = clock64();
      while (true) {
        if (__all_sync(0xffffffffu, mbar_try_wait(&sm.full[s], ph))) break;
        try_drain();
        if (clock64() - t0 > 4000000000LL) {
          if (lane == 0) atomicCAS(sm.status, 0, 2);
          failed = true;
          break;
        }
      }
      if (failed) break;
      const int64_t y = r_begin + static_cast<int64_t>(kb) * kKB;
      const int64_t left = r_end - y;
      const int valid = left < kKB ? static_cast<int>(left) : kKB;
      if (valid == kKB) {
        split_tile<kGramSplitThreads>(sm.a_hi(s), sm.a_lo(s), kABytes / 16, tid);
        split_tile<kGramSplitThreads>(sm.b_hi(s), sm.b_lo(s), kBBytes / 16, tid);
      } else {
        split_tile_rows<kGramSplitThreads>(sm.a_hi(s), sm.a_lo(s), kABytes / 16, tid, valid);
        split_tile_rows<kGramSplitThreads>(sm.b_hi(s), sm.b_lo(s), kBBytes / 16, tid, valid);
      }
      fence_proxy_async();
      __syncwarp();
      if (lane == 0) mbar_arrive(&sm.split[s]);
      try_drain();
    }
    while (!failed && drained < nsub) {
      if (!__all_sync(0xffffffffu,
                      mbar_wait(&sm.sub_full[drained & 1], (drained >> 1) & 1, 4, sm.status))) {
        failed = true;
        break;
      }
      tc_fence_after();
      drain(drained);
      ++drained;
    }
    // Epilogue: TMEM lane = output row i (within the k tile), column = j, from the
    // running sum.
    if (!failed) {
      tc_fence_after();
      const int i = i0 + q * 32 + lane - sx;  // caller's column index in X
      float* out = partial + static_cast<int64_t>(blockIdx.y) * k * m;
      for (int c = c0; c < c0 + kN / 2; c += 16) {
        float v[16];
        tmem_ld16(lane_base + t2col(c), v);
        if (i >= 0 && i < k) {
#pragma unroll
          for (int e = 0; e < 16; ++e) {
            const int j = j0 + c + e - sy;
            if (j >= 0 && j < m) out[static_cast<int64_t>(j) * k + i] = v[e];
          }
        }
      }
    }
  }
  epilogue_dealloc(sm, warp, tmem, kGramTmemCols);
}

// With `symmetric` (X^T X: k == m, equal column shift `shift`), entries of tiles
// that lie wholly below the diagonal were not computed and read their mirror.
__global__ void gram_tc_reduce(const float* __restrict__ partial, int chunks, int k, int m,
                               double* __restrict__ G, int64_t ldg, int symmetric, int shift) {
  const int64_t idx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t total = static_cast<int64_t>(k) * m;
  if (idx >= total) return;
  const int i = static_cast<int>(idx % k), j = static_cast<int>(idx / k);
  int64_t src = idx;
  if (symmetric && ((i + shift) / kM) * kM >= ((j + shift) / kN) * kN + kN)
    src = static_cast<int64_t>(i) * k + j;
  double s = 0.0;
  for (int c = 0; c < chunks; ++c) s += static_cast<double>(partial[c * total + src]);
  G[static_cast<int64_t>(j) * ldg + i] = s;
}

// --------------------------------------------------------------- Rotation ----
// grid.x = m tiles, grid.y = row tiles. A = X (K-major 128 rows x 32), B = C^T
// split into hi/lo FP32 arrays of m_pad rows x k_pad (K-major, prepared by
// rotate_prep_kernel).
__global__ void __launch_bounds__(kThreads, 1)
rotate_tc_kernel(const __grid_constant__ CUtensorMap tmX, const __grid_constant__ CUtensorMap tmCh,
                 const __grid_constant__ CUtensorMap tmCl, int64_t n, int k, int m, int m_tiles,
                 float* __restrict__ Y, int64_t ldy, float alpha, float beta, int use_beta,
                 int vec_store, int upper_tri, int* status) {
  extern __shared__ uint8_t dyn_smem[];
  const Smem sm = carve(dyn_smem, status);
  const int warp = threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  const int j0 = static_cast<int>(blockIdx.x % m_tiles) * kN;
  const int64_t r0 = static_cast<int64_t>(blockIdx.x / m_tiles) * kM;
  // With an upper-triangular C (CholQR's R^-1), rows k >= j0 + kN of C are zero for
  // this tile's columns: those K blocks contribute exact zeros and are skipped.
  const int k_eff = upper_tri ? min(k, j0 + kN) : k;
  const int nkb = (k_eff + kKB - 1) / kKB;

  prologue(sm, warp);
  const uint32_t tmem = *sm.tmem_slot;

  if (warp == 0 && lane == 0) {
    for (int kb = 0; kb < nkb; ++kb) {
      const int s = kb % kStages;
      const uint32_t ph = (kb / kStages) & 1u;
      if (!mbar_wait(&sm.empty[s], ph ^ 1u, 1, sm.status)) break;
      mbar_expect_tx(&sm.full[s], kABytes + 2 * kBBytes);
      tma_load_2d(sm.a_hi(s), &tmX, kb * kKB, static_cast<int>(r0), &sm.full[s]);
      tma_load_2d(sm.b_hi(s), &tmCh, kb * kKB, j0, &sm.full[s]);
      tma_load_2d(sm.b_lo(s), &tmCl, kb * kKB, j0, &sm.full[s]);
    }
  } else if (warp == 1) {
    if (lane == 0) mma_loop<false>(sm, tmem, nkb, idesc_tf32(false, false));
    __syncwarp();
  } else if (warp >= 2) {
    const int tid = threadIdx.x - 64;
    for (int kb = 0; kb < nkb; ++kb) {
      const int s = kb % kStages;
      const uint32_t ph = (kb / kStages) & 1u;
      if (!__all_sync(0xffffffffu, mbar_wait(&sm.full[s], ph, 2, sm.status))) break;
      split_tile(sm.a_hi(s), sm.a_lo(s), kABytes / 16, tid);
      fence_proxy_async();
      __syncwarp();
      if (lane == 0) mbar_arrive(&sm.split[s]);
    }
    // Epilogue: TMEM lane = tile row, column = output column. A 16-byte aligned Y
    // is written straight from registers, four floats per store along each row.
    // Otherwise (a column view such as V[:, locked:] at any offset) each warp
    // stages its 32 rows x kN slice in the (now idle) pipeline shared memory and
    // writes Y row by row with lanes on consecutive columns, so stores stay
    // coalesced instead of one 4-byte store per row per lane.
    if (vec_store) {
      if (mbar_wait(sm.accum, 0, 4, sm.status)) {
        tc_fence_after();
        const int q = warp % 4;
        const int64_t r = r0 + q * 32 + lane;
        for (int c = 0; c < kN; c += 16) {
          float v[16];
          tmem_ld16(tmem + (static_cast<uint32_t>(q * 32) << 16) + c, v);
          if (r >= n) continue;
          float* yr = Y + r * ldy + j0 + c;
          if (j0 + c + 16 <= m) {
#pragma unroll
            for (int e = 0; e < 16; e += 4) {
              float4 o = make_float4(alpha * v[e], alpha * v[e + 1], alpha * v[e + 2],
                                     alpha * v[e + 3]);
              if (use_beta) {
                const float4 y = *reinterpret_cast<const float4*>(yr + e);
                o.x = fmaf(beta, y.x, o.x);
                o.y = fmaf(beta, y.y, o.y);
                o.z = fmaf(beta, y.z, o.z);
                o.w = fmaf(beta, y.w, o.w);
              }
              *reinterpret_cast<float4*>(yr + e) = o;
            }
          } else {
#pragma unroll
            for (int e = 0; e < 16; ++e) {
              if (j0 + c + e < m) {
                float out = alpha * v[e];
                if (use_beta) out = fmaf(beta, yr[e], out);
                yr[e] = out;
              }
            }
          }
        }
      }
    } else if (mbar_wait(sm.accum, 0, 4, sm.status)) {
      tc_fence_after();
      const int q = warp % 4;
      float* stage = reinterpret_cast<float*>(sm.base) + q * (32 * kStageLd);
      for (int c = 0; c < kN; c += 16) {
        float v[16];
        tmem_ld16(tmem + (static_cast<uint32_t>(q * 32) << 16) + c, v);
#pragma unroll
        for (int e = 0; e < 16; ++e) stage[lane * kStageLd + c + e] = v[e];
      }
      __syncwarp();
      const int jn = min(kN, m - j0);
      for (int rr = 0; rr < 32; ++rr) {
        const int64_t r = r0 + q * 32 + rr;
        if (r >= n) break;
        float* yr = Y + r * ldy + j0;
        for (int c = lane; c < jn; c += 32) {
          float o = alpha * stage[rr * kStageLd + c];
          if (use_beta) o = fmaf(beta, yr[c], o);
          yr[c] = o;
        }
      }
    }
  }
  epilogue_dealloc(sm, warp, tmem);
}

// Persistent variant for 16-byte aligned outputs: one CTA per SM loops over
// tiles (column tile fastest); the operand ring continues across tiles and the
// accumulator alternates between two TMEM buffers, so four dedicated epilogue
// warps drain tile i while the producer, split and MMA warps already run tile
// i+1 (no per-tile prologue, pipeline fill or exposed epilogue). Warps: 0 TMA
// producer, 1 MMA issuer, 2-5 hi/lo split, 6-9 epilogue.
constexpr int kPersistThreads = 320;
constexpr uint32_t kPersistTmemCols = 512;
constexpr uint32_t kAccStride = 256;  // TMEM columns between the two accumulators

__global__ void __launch_bounds__(kPersistThreads, 1)
rotate_tc_persistent_kernel(const __grid_constant__ CUtensorMap tmX,
                            const __grid_constant__ CUtensorMap tmCh,
                            const __grid_constant__ CUtensorMap tmCl, int64_t n, int k, int m,
                            int m_tiles, int64_t total_tiles, float* __restrict__ Y, int64_t ldy,
                            float alpha, float beta, int use_beta, int upper_tri,
                            int* status) {
  extern __shared__ uint8_t dyn_smem[];
  const Smem sm = carve(dyn_smem, status);
  // Accumulator full (MMA -> epilogue) and empty (epilogue -> MMA) barriers, after
  // the TMEM address slot.
  uint64_t* accf = reinterpret_cast<uint64_t*>(sm.tmem_slot + 2);
  uint64_t* acce = accf + 2;
  const int warp = threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&sm.full[s], 1);
      mbar_init(&sm.empty[s], 1);
      mbar_init(&sm.split[s], kSplitThreads / 32);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&accf[b], 1);
      mbar_init(&acce[b], 4);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    fence_proxy_async();
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(sm.tmem_slot)),
                 "r"(kPersistTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *sm.tmem_slot;
  const int nkb_full = (k + kKB - 1) / kKB;
  auto tile_nkb = [&](int j0) {
    return upper_tri ? (min(k, j0 + kN) + kKB - 1) / kKB : nkb_full;
  };

  if (warp == 0) {
    if (lane == 0) {
      uint32_t g = 0;
      bool ok = true;
      for (int64_t t = blockIdx.x; ok && t < total_tiles; t += gridDim.x) {
        const int j0 = static_cast<int>(t % m_tiles) * kN;
        const int r0 = static_cast<int>((t / m_tiles) * kM);
        const int nkb = tile_nkb(j0);
        for (int kb = 0; kb < nkb; ++kb, ++g) {
          const int s = static_cast<int>(g % kStages);
          const uint32_t ph = (g / kStages) & 1u;
          if (!mbar_wait(&sm.empty[s], ph ^ 1u, 1, sm.status)) {
            ok = false;
            break;
          }
          mbar_expect_tx(&sm.full[s], kABytes + 2 * kBBytes);
          tma_load_2d(sm.a_hi(s), &tmX, kb * kKB, r0, &sm.full[s]);
          tma_load_2d(sm.b_hi(s), &tmCh, kb * kKB, j0, &sm.full[s]);
          tma_load_2d(sm.b_lo(s), &tmCl, kb * kKB, j0, &sm.full[s]);
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = idesc_tf32(false, false);
      uint32_t g = 0;
      int lt = 0;
      bool ok = true;
      for (int64_t t = blockIdx.x; ok && t < total_tiles; t += gridDim.x, ++lt) {
        const int j0 = static_cast<int>(t % m_tiles) * kN;
        const int nkb = tile_nkb(j0);
        const int b = lt & 1;
        if (lt >= 2 && !mbar_wait(&acce[b], static_cast<uint32_t>((lt >> 1) - 1) & 1u, 5, sm.status)) break;
        tc_fence_after();
        const uint32_t acc_tmem = tmem + static_cast<uint32_t>(b) * kAccStride;
        for (int kb = 0; kb < nkb; ++kb, ++g) {
          const int s = static_cast<int>(g % kStages);
          const uint32_t ph = (g / kStages) & 1u;
          if (!mbar_wait(&sm.split[s], ph, 3, sm.status)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t ah = smem_u32(sm.a_hi(s)), al = smem_u32(sm.a_lo(s));
          const uint32_t bh = smem_u32(sm.b_hi(s)), bl = smem_u32(sm.b_lo(s));
#pragma unroll
          for (int kk = 0; kk < kKB / 8; ++kk) {
            const uint32_t off = kk * 32u;
            const uint64_t dah = smem_desc(ah + off, 16u, 1024u, kLayoutSW128);
            const uint64_t dal = smem_desc(al + off, 16u, 1024u, kLayoutSW128);
            const uint64_t dbh = smem_desc(bh + off, 16u, 1024u, kLayoutSW128);
            const uint64_t dbl = smem_desc(bl + off, 16u, 1024u, kLayoutSW128);
            const uint32_t acc = (kb > 0 || kk > 0) ? 1u : 0u;
            umma_tf32(acc_tmem, dah, dbh, idesc, acc);
            umma_tf32(acc_tmem, dah, dbl, idesc, 1u);
            umma_tf32(acc_tmem, dal, dbh, idesc, 1u);
          }
          umma_commit(&sm.empty[s]);
        }
        if (!ok) break;
        umma_commit(&accf[b]);
      }
    }
    __syncwarp();
  } else if (warp < 6) {
    const int tid = threadIdx.x - 64;
    uint32_t g = 0;
    bool ok = true;
    for (int64_t t = blockIdx.x; ok && t < total_tiles; t += gridDim.x) {
      const int j0 = static_cast<int>(t % m_tiles) * kN;
      const int nkb = tile_nkb(j0);
      for (int kb = 0; kb < nkb; ++kb, ++g) {
        const int s = static_cast<int>(g % kStages);
        const uint32_t ph = (g / kStages) & 1u;
        if (!__all_sync(0xffffffffu, mbar_wait(&sm.full[s], ph, 2, sm.status))) {
          ok = false;
          break;
        }
        split_tile(sm.a_hi(s), sm.a_lo(s), kABytes / 16, tid);
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) mbar_arrive(&sm.split[s]);
      }
    }
  } else {
    const int q = warp % 4;
    int lt = 0;
    for (int64_t t = blockIdx.x; t < total_tiles; t += gridDim.x, ++lt) {
      const int j0 = static_cast<int>(t % m_tiles) * kN;
      const int64_t r0 = (t / m_tiles) * kM;
      const int b = lt & 1;
      if (!mbar_wait(&accf[b], static_cast<uint32_t>(lt >> 1) & 1u, 4, sm.status)) break;
      tc_fence_after();
      const int64_t r = r0 + q * 32 + lane;
      const uint32_t base = tmem + static_cast<uint32_t>(b) * kAccStride +
                            (static_cast<uint32_t>(q * 32) << 16);
      for (int c = 0; c < kN; c += 16) {
        float v[16];
        tmem_ld16(base + c, v);
        if (r >= n) continue;
        float* yr = Y + r * ldy + j0 + c;
        if (j0 + c + 16 <= m) {
#pragma unroll
          for (int e = 0; e < 16; e += 4) {
            float4 o = make_float4(alpha * v[e], alpha * v[e + 1], alpha * v[e + 2],
                                   alpha * v[e + 3]);
            if (use_beta) {
              const float4 y = *reinterpret_cast<const float4*>(yr + e);
              o.x = fmaf(beta, y.x, o.x);
              o.y = fmaf(beta, y.y, o.y);
              o.z = fmaf(beta, y.z, o.z);
              o.w = fmaf(beta, y.w, o.w);
            }
            *reinterpret_cast<float4*>(yr + e) = o;
          }
        } else {
#pragma unroll
          for (int e = 0; e < 16; ++e) {
            if (j0 + c + e < m) {
              float out = alpha * v[e];
              if (use_beta) out = fmaf(beta, yr[e], out);
              yr[e] = out;
            }
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acce[b]);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kPersistTmemCols)
                 : "memory");
  }
}

// C (k x m FP64 column-major) -> Ch, Cl (m_pad x k_pad FP32 row-major = C^T, K-major),
// zero-padded.

// Test probe of the bounded wait: one warp waits on an mbarrier that nothing
// arrives on, for `limit` SM clocks, then records `code` in `status` (or the
// library's default word) and returns. No copies are in flight, so the timeout
// path leaves nothing behind.
// Persistent rotation with X split once in registers and fed to the MMA from tensor
// memory: the split warps read each raw X row of a stage from shared memory (row r of
// the tile = TMEM lane r, one thread per row), round it to hi = rna(x), lo = rna(x - hi)
// and store both into one of two TMEM A slots (32 columns each, in the columns the two
// accumulators leave free), so the MMAs read only C's hi/lo tiles from shared memory.
// Per K stage this moves 132 KB through shared memory where the split in place moves
// 212 KB; the MMAs, their order and so the results are those of
// rotate_tc_persistent_kernel, bit for bit.
// Three A slots (one per pipeline stage), hi and lo 32 columns each, in the TMEM
// columns the accumulators at [0, 160) and [256, 416) leave free.
constexpr int kRotASlots = 3;
__device__ __forceinline__ uint32_t rot_a_hi(int slot) {
  return slot == 0 ? 160u : (slot == 1 ? 224u : 448u);
}
__device__ __forceinline__ uint32_t rot_a_lo(int slot) {
  return slot == 0 ? 192u : (slot == 1 ? 416u : 480u);
}
constexpr int kTmemRotThreads = 448;  // producer, MMA, 8 split warps, 4 epilogue warps

__global__ void __launch_bounds__(kTmemRotThreads, 1)
rotate_tc_tmem_kernel(const __grid_constant__ CUtensorMap tmX,
                      const __grid_constant__ CUtensorMap tmCh,
                      const __grid_constant__ CUtensorMap tmCl, int64_t n, int k, int m,
                      int m_tiles, int64_t total_tiles, float* __restrict__ Y, int64_t ldy,
                      float alpha, float beta, int use_beta, int upper_tri, int* status) {
  extern __shared__ uint8_t dyn_smem[];
  const Smem sm = carve(dyn_smem, status);
  // Accumulator full / empty and A-slot free barriers, after the TMEM address slot.
  uint64_t* accf = reinterpret_cast<uint64_t*>(sm.tmem_slot + 2);
  uint64_t* acce = accf + 2;
  uint64_t* afree = acce + 2;
  const int warp = threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&sm.full[s], 1);
      mbar_init(&sm.empty[s], 1);
      mbar_init(&sm.split[s], 8);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&accf[b], 1);
      mbar_init(&acce[b], 4);
    }
    for (int b = 0; b < kRotASlots; ++b) mbar_init(&afree[b], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    fence_proxy_async();
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(sm.tmem_slot)),
                 "r"(kPersistTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *sm.tmem_slot;
  const int nkb_full = (k + kKB - 1) / kKB;
  auto tile_nkb = [&](int j0) {
    return upper_tri ? (min(k, j0 + kN) + kKB - 1) / kKB : nkb_full;
  };

  if (warp == 0) {
    if (lane == 0) {
      uint32_t g = 0;
      bool ok = true;
      for (int64_t t = blockIdx.x; ok && t < total_tiles; t += gridDim.x) {
        const int j0 = static_cast<int>(t % m_tiles) * kN;
        const int r0 = static_cast<int>((t / m_tiles) * kM);
        const int nkb = tile_nkb(j0);
        for (int kb = 0; kb < nkb; ++kb, ++g) {
          const int s = static_cast<int>(g % kStages);
          const uint32_t ph = (g / kStages) & 1u;
          if (!mbar_wait(&sm.empty[s], ph ^ 1u, 1, sm.status)) {
            ok = false;
            break;
          }
          mbar_expect_tx(&sm.full[s], kABytes + 2 * kBBytes);
          tma_load_2d(sm.a_hi(s), &tmX, kb * kKB, r0, &sm.full[s]);
          tma_load_2d(sm.b_hi(s), &tmCh, kb * kKB, j0, &sm.full[s]);
          tma_load_2d(sm.b_lo(s), &tmCl, kb * kKB, j0, &sm.full[s]);
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = idesc_tf32(false, false);
      uint32_t g = 0;
      int lt = 0;
      bool ok = true;
      for (int64_t t = blockIdx.x; ok && t < total_tiles; t += gridDim.x, ++lt) {
        const int j0 = static_cast<int>(t % m_tiles) * kN;
        const int nkb = tile_nkb(j0);
        const int b = lt & 1;
        if (lt >= 2 &&
            !mbar_wait(&acce[b], static_cast<uint32_t>((lt >> 1) - 1) & 1u, 5, sm.status))
          break;
        tc_fence_after();
        const uint32_t acc_tmem = tmem + static_cast<uint32_t>(b) * kAccStride;
        for (int kb = 0; kb < nkb; ++kb, ++g) {
          const int s = static_cast<int>(g % kStages);
          const uint32_t ph = (g / kStages) & 1u;
          const int slot = static_cast<int>(g % kRotASlots);
          if (!mbar_wait(&sm.split[s], ph, 3, sm.status)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t ahi = tmem + rot_a_hi(slot), alo = tmem + rot_a_lo(slot);
          const uint32_t bh = smem_u32(sm.b_hi(s)), bl = smem_u32(sm.b_lo(s));
#pragma unroll
          for (int kk = 0; kk < kKB / 8; ++kk) {
            const uint32_t a_h = ahi + static_cast<uint32_t>(kk * 8);
            const uint32_t a_l = alo + static_cast<uint32_t>(kk * 8);
            const uint64_t dbh = smem_desc(bh + kk * 32u, 16u, 1024u, kLayoutSW128);
            const uint64_t dbl = smem_desc(bl + kk * 32u, 16u, 1024u, kLayoutSW128);
            const uint32_t acc = (kb > 0 || kk > 0) ? 1u : 0u;
            umma_tf32_ta(acc_tmem, a_h, dbh, idesc, acc);
            umma_tf32_ta(acc_tmem, a_h, dbl, idesc, 1u);
            umma_tf32_ta(acc_tmem, a_l, dbh, idesc, 1u);
          }
          umma_commit(&sm.empty[s]);
          umma_commit(&afree[slot]);
        }
        if (!ok) break;
        umma_commit(&accf[b]);
      }
    }
    __syncwarp();
  } else if (warp < 10) {
    // split warps: warp w owns TMEM lanes 32 (w % 4) .. + 31 = rows of the X tile and
    // half (w - 2) / 4 of the stage's 32 K columns
    const int q = warp % 4;
    const int h = (warp - 2) / 4;
    const int r = q * 32 + lane;
    const uint32_t lane_base = tmem + (static_cast<uint32_t>(q * 32) << 16);
    uint32_t g = 0;
    bool ok = true;
    for (int64_t t = blockIdx.x; ok && t < total_tiles; t += gridDim.x) {
      const int j0 = static_cast<int>(t % m_tiles) * kN;
      const int nkb = tile_nkb(j0);
      for (int kb = 0; kb < nkb; ++kb, ++g) {
        const int s = static_cast<int>(g % kStages);
        const uint32_t ph = (g / kStages) & 1u;
        const int slot = static_cast<int>(g % kRotASlots);
        if (!__all_sync(0xffffffffu, mbar_wait(&sm.full[s], ph, 2, sm.status))) {
          ok = false;
          break;
        }
        if (g >= static_cast<uint32_t>(kRotASlots) &&
            !__all_sync(0xffffffffu,
                        mbar_wait(&afree[slot], ((g / kRotASlots) - 1) & 1u, 6, sm.status))) {
          ok = false;
          break;
        }
        tc_fence_after();
        // row r of the tile: 128 bytes, 16-byte chunk j stored at j ^ (r % 8) (128-byte
        // swizzle of the TMA box); this warp takes chunks 4h .. 4h + 3
        const uint8_t* rowp = reinterpret_cast<const uint8_t*>(sm.a_hi(s)) + r * 128;
        uint32_t hi[16], lo[16];
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
          const int j = 4 * h + jj;
          const float4 v = *reinterpret_cast<const float4*>(rowp + ((j ^ (r & 7)) * 16));
          float4 hv, lv;
          split4(v, hv, lv);
          hi[4 * jj] = __float_as_uint(hv.x);
          hi[4 * jj + 1] = __float_as_uint(hv.y);
          hi[4 * jj + 2] = __float_as_uint(hv.z);
          hi[4 * jj + 3] = __float_as_uint(hv.w);
          lo[4 * jj] = __float_as_uint(lv.x);
          lo[4 * jj + 1] = __float_as_uint(lv.y);
          lo[4 * jj + 2] = __float_as_uint(lv.z);
          lo[4 * jj + 3] = __float_as_uint(lv.w);
        }
        tmem_st16(lane_base + rot_a_hi(slot) + 16u * h, reinterpret_cast<const float*>(hi));
        tmem_st16(lane_base + rot_a_lo(slot) + 16u * h, reinterpret_cast<const float*>(lo));
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&sm.split[s]);
      }
    }
  } else {
    const int q = warp % 4;
    int lt = 0;
    for (int64_t t = blockIdx.x; t < total_tiles; t += gridDim.x, ++lt) {
      const int j0 = static_cast<int>(t % m_tiles) * kN;
      const int64_t r0 = (t / m_tiles) * kM;
      const int b = lt & 1;
      if (!mbar_wait(&accf[b], static_cast<uint32_t>(lt >> 1) & 1u, 4, sm.status)) break;
      tc_fence_after();
      const int64_t r = r0 + q * 32 + lane;
      const uint32_t base = tmem + static_cast<uint32_t>(b) * kAccStride +
                            (static_cast<uint32_t>(q * 32) << 16);
      for (int c = 0; c < kN; c += 16) {
        float v[16];
        tmem_ld16(base + c, v);
        if (r >= n) continue;
        float* yr = Y + r * ldy + j0 + c;
        if (j0 + c + 16 <= m) {
#pragma unroll
          for (int e = 0; e < 16; e += 4) {
            float4 o = make_float4(alpha * v[e], alpha * v[e + 1], alpha * v[e + 2],
                                   alpha * v[e + 3]);
            if (use_beta) {
              const float4 y = *reinterpret_cast<const float4*>(yr + e);
              o.x = fmaf(beta, y.x, o.x);
              o.y = fmaf(beta, y.y, o.y);
              o.z = fmaf(beta, y.z, o.z);
              o.w = fmaf(beta, y.w, o.w);
            }
            *reinterpret_cast<float4*>(yr + e) = o;
          }
        } else {
#pragma unroll
          for (int e = 0; e < 16; ++e) {
            if (j0 + c + e < m) {
              float out = alpha * v[e];
              if (use_beta) out = fmaf(beta, yr[e], out);
              yr[e] = out;
            }
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acce[b]);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kPersistTmemCols)
                 : "memory");
  }
}

__global__ void wait_probe_kernel(int* status, long long limit, int code) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) mbar_wait_limit(&bar, 0, code, status ? status : &g_tc_status, limit);
  __syncthreads();
}

__global__ void rotate_prep_kernel(const double* __restrict__ C, int64_t ldc, int k, int m,
                                   int k_pad, int m_pad, float* __restrict__ Ch,
                                   float* __restrict__ Cl) {
  const int64_t idx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= static_cast<int64_t>(k_pad) * m_pad) return;
  const int kk = static_cast<int>(idx % k_pad);
  const int j = static_cast<int>(idx / k_pad);
  float hi = 0.0f, lo = 0.0f;
  if (kk < k && j < m) {
    const double c = C[static_cast<int64_t>(j) * ldc + kk];
    const float cf = static_cast<float>(c);
    hi = __uint_as_float(tf32_rna(cf));
    lo = __uint_as_float(tf32_rna(static_cast<float>(c - static_cast<double>(hi))));
  }
  Ch[idx] = hi;
  Cl[idx] = lo;
}

// ------------------------------------------------------------ host side ----
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  if (!fn) throw Error(FE_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
  return fn;
}

// 2D FP32 tensor map over rows x cols (row stride ld elements), box box_x x box_y,
// 128-byte swizzle (16-byte chunks for K-major operands, 32-byte chunks for the
// MN-major TF32 operands of the Gram), zero fill out of bounds.
CUtensorMap make_map(const float* base, int64_t cols, int64_t rows, int64_t ld, int box_x,
                     int box_y, bool swizzle_32b_atoms = false) {
  FE_REQUIRE((reinterpret_cast<uintptr_t>(base) & 15u) == 0, "tensor map base not 16-byte aligned");
  FE_REQUIRE((ld * 4) % 16 == 0, "tensor map row stride not a multiple of 16 bytes");
  CUtensorMap map;
  cuuint64_t dims[2] = {static_cast<cuuint64_t>(cols), static_cast<cuuint64_t>(rows)};
  cuuint64_t strides[1] = {static_cast<cuuint64_t>(ld * 4)};
  cuuint32_t box[2] = {static_cast<cuuint32_t>(box_x), static_cast<cuuint32_t>(box_y)};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = encode_fn()(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base),
                           dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           swizzle_32b_atoms ? CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B
                                             : CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw Error(FE_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string(r));
  return map;
}

void set_smem_attr(const void* kernel) {
  FE_CHECK_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     kSmemBytes));
}

constexpr int kGramTcTargetChunks = 384;

struct TcGramPlan {
  int k_tiles, m_tiles, chunks;
  int64_t rows_per_chunk;
  size_t bytes;
};

// Row chunks: as many as make the CTAs that compute (the output tiles, less those
// wholly below the diagonal of a symmetric Gram) fill two whole waves of one CTA per
// SM, so every SM gets equal work, the per-CTA prologue and partial tile are paid a few
// hundred times rather than thousands, and no tail wave runs half empty; at least four
// K stages per chunk.
TcGramPlan tc_gram_plan(int64_t n, int64_t kx, int64_t my, int64_t k, int64_t m,
                        int64_t active_tiles) {
  TcGramPlan p{};
  p.k_tiles = static_cast<int>((kx + kM - 1) / kM);
  p.m_tiles = static_cast<int>((my + kN - 1) / kN);
  const int64_t tiles = std::max<int64_t>(1, active_tiles);
  int64_t chunks = std::max<int64_t>(1, (2 * static_cast<int64_t>(num_sms())) / tiles);
  chunks = std::min<int64_t>({chunks, kGramTcTargetChunks, (n + 4 * kKB - 1) / (4 * kKB)});
  chunks = std::max<int64_t>(chunks, 1);
  int64_t rpc = (n + chunks - 1) / chunks;
  rpc = ((rpc + kKB - 1) / kKB) * kKB;
  p.rows_per_chunk = rpc;
  p.chunks = static_cast<int>((n + rpc - 1) / rpc);
  p.bytes = static_cast<size_t>(p.chunks) * k * m * sizeof(float);
  return p;
}

}  // namespace

bool tc_gemm_available() {
  static int ok = -1;
  if (ok < 0) {
    int dev = 0, major = 0, minor = 0;
    ok = (cudaGetDevice(&dev) == cudaSuccess &&
          cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) == cudaSuccess &&
          cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev) == cudaSuccess &&
          major == 10 && minor == 0)
             ? 1
             : 0;
  }
  return ok == 1;
}

size_t tc_gram_workspace_bytes(int64_t n, int64_t k, int64_t m) {
  if (n <= 0 || k <= 0 || m <= 0) return 0;
  // bound over every call with n' <= n, k' <= k, m' <= m (chunk count <= target)
  const int64_t chunks = std::min<int64_t>(kGramTcTargetChunks, (n + 4 * kKB - 1) / (4 * kKB));
  return static_cast<size_t>(std::max<int64_t>(chunks, 1)) * k * m * sizeof(float);
}

// G = X^T Y (FP32 inputs, 3xTF32 tensor cores, FP64 reduction of chunk partials).
void gram_tc(const float* X, int64_t ldx, const float* Y, int64_t ldy, int64_t n, int64_t k,
             int64_t m, double* G, int64_t ldg, void* ws, size_t ws_bytes, cudaStream_t s) {
  FE_REQUIRE(n > 0 && k > 0 && m > 0 && ldg >= k, "gram_tc: invalid shape");
  FE_REQUIRE(n < (int64_t(1) << 31), "gram_tc: too many rows for 32-bit TMA coordinates");
  const int sx = static_cast<int>((reinterpret_cast<uintptr_t>(X) & 15u) / 4);
  const int sy = static_cast<int>((reinterpret_cast<uintptr_t>(Y) & 15u) / 4);
  const float* Xa = X - sx;
  const float* Ya = Y - sy;
  const bool sym = X == Y && ldx == ldy && k == m;
  int64_t active_tiles = 0;
  {
    const int64_t kt = (k + sx + kM - 1) / kM, mt = (m + sy + kN - 1) / kN;
    for (int64_t ti = 0; ti < kt; ++ti)
      for (int64_t tj = 0; tj < mt; ++tj)
        if (!(sym && ti * kM >= tj * kN + kN)) ++active_tiles;
  }
  const TcGramPlan p = tc_gram_plan(n, k + sx, m + sy, k, m, active_tiles);
  FE_REQUIRE(ws && ws_bytes >= p.bytes, "gram_tc: workspace too small");
  const CUtensorMap mx = make_map(Xa, k + sx, n, ldx, 32, kKB, true);
  const CUtensorMap my = make_map(Ya, m + sy, n, ldy, 32, kKB, true);
  static std::once_flag once;
  std::call_once(once, [] { set_smem_attr(reinterpret_cast<const void*>(gram_tc_kernel)); });
  dim3 grid(p.k_tiles * p.m_tiles, p.chunks);
  gram_tc_kernel<<<grid, kGramThreads, kSmemBytes, s>>>(mx, my, n, static_cast<int>(k),
                                                    static_cast<int>(m), sx, sy, p.k_tiles,
                                                    p.rows_per_chunk, static_cast<float*>(ws),
                                                    sym ? 1 : 0, current_status_word());
  check_launch("gram_tc_kernel");
  const int64_t total = k * m;
  gram_tc_reduce<<<static_cast<unsigned>((total + 255) / 256), 256, 0, s>>>(
      static_cast<const float*>(ws), p.chunks, static_cast<int>(k), static_cast<int>(m), G, ldg,
      sym ? 1 : 0, sx);
  check_launch("gram_tc_reduce");
}

size_t tc_rotate_workspace_bytes(int64_t k, int64_t m) {
  if (k <= 0 || m <= 0) return 0;
  const int64_t k_pad = ((k + kKB - 1) / kKB) * kKB;
  const int64_t m_pad = ((m + kN - 1) / kN) * kN;
  return static_cast<size_t>(2 * k_pad * m_pad) * sizeof(float);
}

// Y = alpha X C + beta Y (FP32 blocks, 3xTF32 tensor cores).
void rotate_tc(const float* X, int64_t ldx, const double* C, int64_t ldc, float* Y, int64_t ldy,
               int64_t n, int64_t k, int64_t m, double alpha, double beta, void* ws,
               size_t ws_bytes, cudaStream_t s, bool upper_tri) {
  FE_REQUIRE(n > 0 && k > 0 && m > 0, "rotate_tc: invalid shape");
  FE_REQUIRE(n < (int64_t(1) << 31), "rotate_tc: too many rows for 32-bit TMA coordinates");
  FE_REQUIRE((reinterpret_cast<uintptr_t>(X) & 15u) == 0, "rotate_tc: X not 16-byte aligned");
  const int64_t k_pad = ((k + kKB - 1) / kKB) * kKB;
  const int64_t m_pad = ((m + kN - 1) / kN) * kN;
  FE_REQUIRE(ws && ws_bytes >= tc_rotate_workspace_bytes(k, m), "rotate_tc: workspace too small");
  float* Ch = static_cast<float*>(ws);
  float* Cl = Ch + k_pad * m_pad;
  const int64_t total = k_pad * m_pad;
  rotate_prep_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, s>>>(
      C, ldc, static_cast<int>(k), static_cast<int>(m), static_cast<int>(k_pad),
      static_cast<int>(m_pad), Ch, Cl);
  check_launch("rotate_prep_kernel");
  const CUtensorMap mx = make_map(X, k, n, ldx, kKB, kM);
  const CUtensorMap mh = make_map(Ch, k_pad, m_pad, k_pad, kKB, kN);
  const CUtensorMap ml = make_map(Cl, k_pad, m_pad, k_pad, kKB, kN);
  static std::once_flag once;
  std::call_once(once, [] { set_smem_attr(reinterpret_cast<const void*>(rotate_tc_kernel)); });
  const int64_t row_tiles = (n + kM - 1) / kM;
  const int64_t m_tiles = m_pad / kN;
  FE_REQUIRE(row_tiles * m_tiles <= 2147483647LL, "rotate_tc: too many tiles");
  const bool vec = (reinterpret_cast<uintptr_t>(Y) & 15u) == 0 && ldy % 4 == 0;
  const int64_t total_tiles = row_tiles * m_tiles;
  if (vec && g_rotate_persistent) {
    static std::once_flag once_p;
    std::call_once(once_p, [] {
      FE_CHECK_CUDA(cudaFuncSetAttribute(rotate_tc_persistent_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kSmemBytes));
      FE_CHECK_CUDA(cudaFuncSetAttribute(rotate_tc_tmem_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kSmemBytes));
    });
    const int64_t ctas = std::min<int64_t>(total_tiles, num_sms());
    const bool tmem_a = g_rotate_persistent == 2;
    auto kern = tmem_a ? rotate_tc_tmem_kernel : rotate_tc_persistent_kernel;
    kern<<<static_cast<unsigned>(ctas), tmem_a ? kTmemRotThreads : kPersistThreads, kSmemBytes,
           s>>>(
        mx, mh, ml, n, static_cast<int>(k), static_cast<int>(m), static_cast<int>(m_tiles),
        total_tiles, Y, ldy, static_cast<float>(alpha), static_cast<float>(beta), beta != 0.0,
        upper_tri ? 1 : 0, current_status_word());
    check_launch(g_rotate_persistent == 2 ? "rotate_tc_tmem_kernel"
                                          : "rotate_tc_persistent_kernel");
    return;
  }
  dim3 grid(static_cast<unsigned>(row_tiles * m_tiles));
  rotate_tc_kernel<<<grid, kThreads, kSmemBytes, s>>>(mx, mh, ml, n, static_cast<int>(k),
                                                      static_cast<int>(m),
                                                      static_cast<int>(m_tiles), Y, ldy,
                                                      static_cast<float>(alpha),
                                                      static_cast<float>(beta), beta != 0.0,
                                                      vec ? 1 : 0, upper_tri ? 1 : 0,
                                                      current_status_word());
  check_launch("rotate_tc_kernel");
}

void launch_wait_probe(int* status, long long limit_cycles, int code, cudaStream_t s) {
  wait_probe_kernel<<<1, 32, 0, s>>>(status, limit_cycles, code);
  check_launch("wait_probe_kernel");
}

int read_tc_status(bool clear) {
  int v = 0;
  FE_CHECK_CUDA(cudaMemcpyFromSymbol(&v, g_tc_status, sizeof(int)));
  if (clear && v != 0) {
    const int z = 0;
    FE_CHECK_CUDA(cudaMemcpyToSymbol(g_tc_status, &z, sizeof(int)));
  }
  return v;
}

}  // namespace fe

extern "C" int fe_selftest_wait_timeout(int64_t limit_cycles, int32_t code, void* stream) {
  return fe::guarded("fe_selftest_wait_timeout", [&] {
    FE_REQUIRE(code != 0, "code must be nonzero");
    FE_REQUIRE(limit_cycles >= 0 && limit_cycles <= 4000000000LL, "limit out of range");
    fe::launch_wait_probe(nullptr, limit_cycles, code, fe::as_stream(stream));
  });
}

extern "C" int fe_device_status(int32_t* status, int32_t clear) {
  return fe::guarded("fe_device_status", [&] {
    FE_REQUIRE(status, "null status");
    const int a = fe::read_tc_status(clear != 0);
    const int b = fe::read_spmm_status(clear != 0);
    *status = a != 0 ? a : b;
  });
}

extern "C" int fe_set_spmm_kernel(int32_t mode) {
  return fe::guarded("fe_set_spmm_kernel", [&] {
    FE_REQUIRE(mode >= 0 && mode <= 7, "mode must be 0..7");
    fe::set_spmm_mode(mode);
  });
}

extern "C" int fe_set_cheb_wave_kernel(int32_t mode) {
  return fe::guarded("fe_set_cheb_wave_kernel", [&] {
    const bool panels = mode >= 100 && (mode / 100 == 1 || mode / 100 == 2 || mode / 100 == 4) &&
                        mode % 100 >= 1 && mode % 100 <= 8;
    FE_REQUIRE((mode >= 0 && mode <= 9) || (mode >= 12 && mode <= 18) || panels,
               "mode must be 0..9, 12..18 or 100 P + S (P in 1, 2, 4; S in 1..8)");
    fe::set_wave_mode(mode);
  });
}

extern "C" int fe_set_tc_rotate_kernel(int32_t mode) {
  return fe::guarded("fe_set_tc_rotate_kernel", [&] {
    FE_REQUIRE(mode >= 0 && mode <= 2, "mode must be 0, 1 or 2");
    // 0: persistent, X split in registers into TMEM; 1: one CTA per tile; 2: persistent,
    // X split in shared memory
    fe::set_rotate_persistent(mode == 0 ? 2 : (mode == 1 ? 0 : 1));
  });
}

extern "C" int fe_set_f64_gemm_kernel(int32_t mode) {
  return fe::guarded("fe_set_f64_gemm_kernel", [&] {
    FE_REQUIRE(mode >= 0 && mode <= 1, "mode must be 0 or 1");
    fe::set_f64_gemm_mode(mode);
  });
}

extern "C" size_t fe_gram_tf32x3_workspace_bytes(int64_t n, int64_t k, int64_t m) {
  return fe::tc_gram_workspace_bytes(n, k, m);
}

extern "C" int fe_gram_tf32x3(const float* X, int64_t ldx, const float* Y, int64_t ldy, int64_t n,
                              int64_t k, int64_t m, double* G, int64_t ldg, void* workspace,
                              size_t workspace_bytes, void* stream) {
  return fe::guarded("fe_gram_tf32x3", [&] {
    FE_REQUIRE(fe::tc_gemm_available(), "tcgen05 kernels need an sm_100 device");
    FE_REQUIRE(X && Y && ldx >= k && ldy >= m, "invalid input block");
    FE_REQUIRE(ldx % 4 == 0 && ldy % 4 == 0, "leading dimensions must be multiples of 4");
    fe::gram_tc(X, ldx, Y, ldy, n, k, m, G, ldg, workspace, workspace_bytes,
                fe::as_stream(stream));
  });
}

extern "C" size_t fe_rotate_tf32x3_workspace_bytes(int64_t k, int64_t m) {
  return fe::tc_rotate_workspace_bytes(k, m);
}

extern "C" int fe_rotate_tf32x3(const float* X, int64_t ldx, const double* C, int64_t ldc,
                                float* Y, int64_t ldy, int64_t n, int64_t k, int64_t m,
                                double alpha, double beta, void* workspace,
                                size_t workspace_bytes, void* stream) {
  return fe::guarded("fe_rotate_tf32x3", [&] {
    FE_REQUIRE(fe::tc_gemm_available(), "tcgen05 kernels need an sm_100 device");
    FE_REQUIRE(X && C && Y && ldx >= k && ldc >= k && ldy >= m, "invalid arguments");
    FE_REQUIRE(ldx % 4 == 0, "ldx must be a multiple of 4");
    FE_REQUIRE(!fe::ranges_overlap(X, n, ldx, k, static_cast<const float*>(Y), n, ldy, m),
               "X and Y overlap");
    fe::rotate_tc(X, ldx, C, ldc, Y, ldy, n, k, m, alpha, beta, workspace, workspace_bytes,
                  fe::as_stream(stream), false);
  });
}
