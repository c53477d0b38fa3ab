// Host-side helpers of the B200 backend: device buffers, row-major block views,
// the kernel entry points shared across translation units, and small host
// dense routines (symmetric Jacobi eigensolver for the Lanczos tridiagonal).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "fe_common.cuh"

namespace fe {

// ---- kernels (defined in spmm.cu / blocks.cu / dense.cu) -----------------
template <typename T>
void csr_spmm(const Csr& A, const T* X, int64_t ldx, T* Y, int64_t ldy, const T* Z, int64_t ldz,
              int64_t ncols, double alpha, double gamma, double beta, cudaStream_t s);
// Refined filter pieces (spmm.cu): the FP32 Chebyshev step with a correction term
// R diag(delta), and the elementwise start (R32 = R64 - X diag(theta), Z1 = c R32) and
// finish (X = X diag(t) + Z) of the correction recurrence.
void csr_spmm_corr_f32(const Csr& A, const float* X, int64_t ldx, float* Y, int64_t ldy,
                       const float* Z, int64_t ldz, const float* R, int64_t ldr,
                       const float* delta, int64_t ncols, double alpha, double gamma, double beta,
                       cudaStream_t s);
void refine_start(int64_t n, int64_t ncols, const double* R64, int64_t ld64, const double* X,
                  int64_t ldx, const double* theta, double c, float* R32, float* Z1,
                  int64_t ld32, cudaStream_t s);
void refine_finish(int64_t n, int64_t ncols, const double* t, const float* Z, int64_t ld32,
                   double* X, int64_t ldx, cudaStream_t s);
template <typename T>
void cheb_filter(const Csr& A, T* X, T* scratch, int64_t ld, int64_t ncols, int degree, double c,
                 double d, cudaStream_t s);
// The filter in launches of several steps each (the result in X, Sc scratch); false
// (nothing launched) where it does not apply. `sync` holds wave_sync_bytes(A.rows).
size_t wave_sync_bytes(int64_t nrows);
void set_wave_mode(int mode);
int64_t csr_bandwidth(const Csr& A, cudaStream_t s);
template <typename T>
bool cheb_filter_wave(const Csr& A, T* X, int64_t ldx, T* Sc, int64_t lds, int64_t ncols,
                      int degree, double c, double d, void* sync, size_t sync_bytes,
                      cudaStream_t s);
size_t gram_workspace_bytes(int64_t n, int64_t k, int64_t m);
template <typename T>
void gram(const T* X, int64_t ldx, const T* Y, int64_t ldy, int64_t n, int64_t k, int64_t m,
          double* G, int64_t ldg, void* ws, size_t ws_bytes, cudaStream_t s);
// upper_tri: C is upper triangular (zero below its diagonal), so the products of
// its zero rows may be skipped.
template <typename T>
void rotate(const T* X, int64_t ldx, const double* C, int64_t ldc, T* Y, int64_t ldy, int64_t n,
            int64_t k, int64_t m, double alpha, double beta, cudaStream_t s,
            bool upper_tri = false);
size_t residual_workspace_bytes(int64_t n, int64_t m);
template <typename T>
void residual_norms(const T* AX, const T* X, const T* BX, int64_t ld, int64_t n, int64_t m,
                    const double* lambda, T* R, int64_t ldr, double* rnorm, double* xnorm,
                    double* rel, void* ws, size_t ws_bytes, cudaStream_t s, int mode);
template <typename S, typename D>
void convert(const S* src, int64_t lds, D* dst, int64_t ldd, int64_t n, int64_t m, cudaStream_t s);
void potrf_upper(double* G, int64_t k, int64_t ldg, int32_t* info, cudaStream_t s);
void trinv_upper(const double* R, int64_t ldr, double* Rinv, int64_t ldi, int64_t k,
                 cudaStream_t s);
void symmetrize(double* P, int64_t k, int64_t ldp, cudaStream_t s);
// Batched k x k forms (grouped solves): `count` matrices `stride` doubles apart.
void potrf_upper_batched(double* G, int64_t k, int64_t ldg, int64_t stride, int64_t count,
                         int32_t* info, cudaStream_t s);
void trinv_upper_batched(const double* R, int64_t ldr, double* Rinv, int64_t ldi, int64_t k,
                         int64_t stride, int64_t count, cudaStream_t s);
void symmetrize_batched(double* P, int64_t k, int64_t ldp, int64_t stride, int64_t count,
                        cudaStream_t s);
// Cholesky and upper-triangular inverse in one launch for k <= 128 (one CTA per
// matrix, shared memory): Rinv = chol(G)^{-1}; info[p] = first failed pivot + 1 or 0.
bool chol_inv_small_fits(int64_t k);
void chol_inv_upper_batched(const double* G, int64_t k, int64_t ldg, int64_t stride_g,
                            double* Rinv, int64_t ldi, int64_t stride_i, int64_t count,
                            int32_t* info, cudaStream_t s);
// Y32 = float(Y), E32 = float(AY - Y diag(theta)) (n x k row-major blocks), and
// H = G diag(theta) + H1 (k x k column-major, leading dimension ld).
void shift_split(int64_t n, int64_t k, const double* AY, int64_t lday, const double* Y,
                 int64_t ldy, const double* theta, float* Y32, float* E32, int64_t ld32,
                 cudaStream_t s);
void gram_shift_combine(int64_t k, int64_t ld, const double* G, const double* theta,
                        const double* H1, double* H, cudaStream_t s);
// Small column-major FP64 products: C = alpha op(A) B + beta C, op(A) = A or A^T.
void small_gemm(bool trans_a, int64_t m, int64_t n, int64_t kk, double alpha, const double* A,
                int64_t lda, const double* B, int64_t ldb, double beta, double* C, int64_t ldc,
                cudaStream_t s);
// d[j] = 1/sqrt(G[j,j]); M <- D M D (both) or D M (rows only).
void inv_sqrt_diag(const double* G, int64_t k, int64_t ldg, double* d, cudaStream_t s);
void diag_scale(double* M, int64_t rows, int64_t cols, int64_t ldm, const double* d, bool both,
                cudaStream_t s);
// Device symmetric eigensolver (syevd.cu): A (k x k, lda, column-major) is replaced
// by its eigenvectors, W gets the ascending eigenvalues, *info (device) is nonzero
// for non-finite input.
size_t syevd_single_workspace_bytes(int64_t k);
void syevd_single(double* A, int64_t lda, int64_t k, double* W, int32_t* info, void* ws,
                  size_t ws_bytes, cudaStream_t s);
// Batched form: `count` matrices A + p*lda*lda of sizes m_host[p] <= lda; eigenvalues
// to W + p*lda, eigenvectors to Z + p*lda*lda; A is overwritten by reflectors.
size_t syevd_workspace_bytes(int count, int64_t lda);
void syevd_batched(int count, const int32_t* m_host, double* A, int64_t lda, double* W,
                   double* Z, int32_t* info, void* ws, size_t ws_bytes, cudaStream_t s);
// Batched form with every matrix of size k and no host-to-device copy (capturable).
void syevd_batched_uniform(int count, int64_t k, double* A, int64_t lda, double* W, double* Z,
                           int32_t* info, void* ws, size_t ws_bytes, cudaStream_t s);

// ---- owning device buffer --------------------------------------------------
// Stream on which this thread's DeviceBuffer allocations are ordered (set for the
// lifetime of a solver Context). With a stream, buffers come from the device's
// stream-ordered memory pool (cudaMallocAsync / cudaFreeAsync), which keeps the
// memory of one solve for the next instead of mapping and unmapping tens of GB
// per solve; without one, plain cudaMalloc / cudaFree.
cudaStream_t& alloc_stream();
// Keep freed pool memory reserved for this process (called once per device).
void retain_pool_memory(int device);
// Large blocks (>= 64 MiB) of a solve: exact-size reuse across solves (see dense.cu).
void* big_alloc(size_t bytes, cudaStream_t s, size_t* granted);
// Frees the cached solve blocks and trims the stream-ordered pool of `device`.
void release_cached_memory(int device);
void big_free(void* p, size_t granted, cudaStream_t s);
constexpr size_t kBigBlockBytes = size_t(64) << 20;

class DeviceBuffer {
 public:
  DeviceBuffer() = default;
  explicit DeviceBuffer(size_t bytes) { resize(bytes); }
  ~DeviceBuffer() { release(); }
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  DeviceBuffer(DeviceBuffer&& o) noexcept
      : p_(o.p_), bytes_(o.bytes_), granted_(o.granted_), s_(o.s_) {
    o.p_ = nullptr;
    o.bytes_ = 0;
    o.granted_ = 0;
    o.s_ = nullptr;
  }
  DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
    if (this != &o) {
      release();
      p_ = o.p_;
      bytes_ = o.bytes_;
      granted_ = o.granted_;
      s_ = o.s_;
      o.p_ = nullptr;
      o.bytes_ = 0;
      o.granted_ = 0;
      o.s_ = nullptr;
    }
    return *this;
  }
  void resize(size_t bytes) {
    if (bytes <= bytes_ && p_) return;
    release();
    if (bytes == 0) return;
    s_ = alloc_stream();
    if (s_ && bytes >= kBigBlockBytes) {
      p_ = big_alloc(bytes, s_, &granted_);
      bytes_ = bytes;
      return;
    }
    cudaError_t e = s_ ? cudaMallocAsync(&p_, bytes, s_) : cudaMalloc(&p_, bytes);
    if (e != cudaSuccess) {
      // give back what the caches hold and try once more
      cudaGetLastError();
      int dev = 0;
      if (cudaGetDevice(&dev) == cudaSuccess) release_cached_memory(dev);
      e = s_ ? cudaMallocAsync(&p_, bytes, s_) : cudaMalloc(&p_, bytes);
    }
    if (e != cudaSuccess) {
      p_ = nullptr;
      throw Error(FE_ERR_ALLOC, std::string("cudaMalloc(") + std::to_string(bytes) +
                                    ") failed: " + cudaGetErrorString(e));
    }
    bytes_ = bytes;
  }
  void release() {
    if (p_) {
      if (granted_) big_free(p_, granted_, s_);
      else if (s_) cudaFreeAsync(p_, s_);
      else cudaFree(p_);
    }
    p_ = nullptr;
    bytes_ = 0;
    granted_ = 0;
    s_ = nullptr;
  }
  void* get() const { return p_; }
  size_t bytes() const { return bytes_; }
  template <typename T>
  T* as() const {
    return static_cast<T*>(p_);
  }

 private:
  void* p_ = nullptr;
  size_t bytes_ = 0;
  size_t granted_ = 0;        // size of a cached large block (0: pool or plain allocation)
  cudaStream_t s_ = nullptr;  // allocation stream (pool / cache) or null (cudaMalloc)
};

// Row-major n-by-cols block with leading dimension ld (padded to 8 elements so
// every row starts 16-byte aligned for vector loads and TMA tiles).
template <typename T>
struct Block {
  DeviceBuffer buf;
  int64_t n = 0, cols = 0, ld = 0;
  void allocate(int64_t rows, int64_t c) {
    n = rows;
    cols = c;
    ld = std::max<int64_t>(8, ((c + 7) / 8) * 8);
    buf.resize(static_cast<size_t>(n) * ld * sizeof(T));
  }
  T* data() const { return buf.as<T>(); }
  T* col(int64_t j) const { return buf.as<T>() + j; }
};

// ---- host small dense -----------------------------------------------------
// Cyclic Jacobi eigensolver for a small symmetric matrix (column-major m-by-m).
// Returns ascending eigenvalues; Z (column-major) holds the eigenvectors.
inline void host_symmetric_eig(std::vector<double> A, int m, std::vector<double>& w,
                               std::vector<double>& Z) {
  Z.assign(static_cast<size_t>(m) * m, 0.0);
  for (int i = 0; i < m; ++i) Z[static_cast<size_t>(i) * m + i] = 1.0;
  auto a = [&](int r, int c) -> double& { return A[static_cast<size_t>(c) * m + r]; };
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, diag = 0.0;
    for (int c = 0; c < m; ++c)
      for (int r = 0; r < m; ++r) (r == c ? diag : off) += a(r, c) * a(r, c);
    if (off <= 1e-30 * std::max(diag, 1e-300)) break;
    for (int p = 0; p < m - 1; ++p) {
      for (int q = p + 1; q < m; ++q) {
        const double apq = a(p, q);
        if (apq == 0.0) continue;
        const double theta = (a(q, q) - a(p, p)) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) /
                         (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0);
        const double s = t * c;
        for (int k = 0; k < m; ++k) {  // columns p, q
          const double akp = a(k, p), akq = a(k, q);
          a(k, p) = c * akp - s * akq;
          a(k, q) = s * akp + c * akq;
        }
        for (int k = 0; k < m; ++k) {  // rows p, q
          const double apk = a(p, k), aqk = a(q, k);
          a(p, k) = c * apk - s * aqk;
          a(q, k) = s * apk + c * aqk;
        }
        for (int k = 0; k < m; ++k) {
          double& zp = Z[static_cast<size_t>(p) * m + k];
          double& zq = Z[static_cast<size_t>(q) * m + k];
          const double zkp = zp, zkq = zq;
          zp = c * zkp - s * zkq;
          zq = s * zkp + c * zkq;
        }
      }
    }
  }
  std::vector<int> order(m);
  for (int i = 0; i < m; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return a(x, x) < a(y, y); });
  w.resize(m);
  std::vector<double> Zs(static_cast<size_t>(m) * m);
  for (int j = 0; j < m; ++j) {
    w[j] = a(order[j], order[j]);
    std::memcpy(&Zs[static_cast<size_t>(j) * m], &Z[static_cast<size_t>(order[j]) * m],
                sizeof(double) * m);
  }
  Z.swap(Zs);
}

}  // namespace fe

namespace fe {
void vec_axpby(int64_t n, double a, const double* x, int64_t incx, double b, double* y,
               int64_t incy, cudaStream_t s);
// y[i*incy] = x[i] / *nrm (divisor on the device); *out = *a + *b (one thread).
void scale_by_inv(int64_t n, const double* x, const double* nrm, double* y, int64_t incy,
                  cudaStream_t s);
void sum2(const double* a, const double* b, double* out, cudaStream_t s);
template <typename T>
void fill_uniform(T* X, int64_t ld, int64_t n, int64_t m, uint64_t seed, cudaStream_t s);
}  // namespace fe

namespace fe {
bool tc_gemm_available();
size_t tc_gram_workspace_bytes(int64_t n, int64_t k, int64_t m);
void gram_tc(const float* X, int64_t ldx, const float* Y, int64_t ldy, int64_t n, int64_t k,
             int64_t m, double* G, int64_t ldg, void* ws, size_t ws_bytes, cudaStream_t s);
size_t tc_rotate_workspace_bytes(int64_t k, int64_t m);
void rotate_tc(const float* X, int64_t ldx, const double* C, int64_t ldc, float* Y, int64_t ldy,
               int64_t n, int64_t k, int64_t m, double alpha, double beta, void* ws,
               size_t ws_bytes, cudaStream_t s, bool upper_tri = false);
int read_tc_status(bool clear);
}  // namespace fe

namespace fe {
template <typename T>
void gather_columns(const T* src, int64_t lds, const int32_t* idx, int64_t m, T* dst, int64_t ldd,
                    int64_t n, cudaStream_t s, const double* row_scale = nullptr);
void jacobi_inverse_diagonal(const Csr& A, double* t, cudaStream_t s);
void small_gather_scale(const double* src, int64_t lds, int64_t rows, const int32_t* idx,
                        const double* scale, int64_t m, double* dst, int64_t ldd, cudaStream_t s);
void mirror_block(double* P, int64_t ld, int64_t rows, int64_t c0, int64_t cols, cudaStream_t s);
void to_colmajor(const double* src, int64_t lds, int64_t n, int64_t m, double* dst,
                 cudaStream_t s);
}  // namespace fe

namespace fe {
// ---- batched Krylov-Schur (batch_ks.cu) -----------------------------------
constexpr int kBatchMaxDim = 96;       // largest subspace dimension of the batched engine
constexpr int kBatchChunkRows = 2048;  // rows per reduction chunk (never crosses problems)

struct BatchLayout {
  int32_t num_problems = 0, num_chunks = 0;
  int64_t M = 0;  // leading dimension of the basis rows and of each T / Z / C
  const int32_t* c_prob = nullptr;
  const int64_t* c_row0 = nullptr;
  const int32_t* c_rows = nullptr;
  const int32_t* p_chunk0 = nullptr;
  const int32_t* p_nchunks = nullptr;
};

struct BatchState {
  int32_t *col = nullptr, *mdim = nullptr, *restart_row = nullptr, *active = nullptr,
          *status = nullptr;
  double *beta = nullptr, *inv = nullptr, *beta_next = nullptr, *T = nullptr, *part = nullptr,
         *part1 = nullptr, *h1 = nullptr, *h2 = nullptr;
};

void bks_lanczos_step(const BatchLayout& L, const BatchState& S, const Csr& A, double* V,
                      int64_t ldv, double* f, double* q, double* w, cudaStream_t s);
void bks_init_norm(const BatchLayout& L, const BatchState& S, const double* f, cudaStream_t s);
void bks_jacobi(const BatchLayout& L, const double* T, const int32_t* mdim, const int32_t* todo,
                int max_m, double* W, double* Z, double* Zlast, cudaStream_t s);
void bks_restart(const BatchLayout& L, const int32_t* mdim, const int32_t* idx,
                 const int32_t* keep, const int32_t* keepY, const double* diag,
                 const double* coup, const double* Z, double* C, double* T, cudaStream_t s);
void bks_rotate(const BatchLayout& L, const double* V, int64_t ldv, const double* C,
                const int32_t* mdim, const int32_t* keep, int max_m, int max_keep, double* dst,
                int64_t ldd, cudaStream_t s);
void bks_residuals(const BatchLayout& L, const int32_t* nev, const double* AY, const double* Y,
                   int64_t ld, const double* lam, int ldl, double* part, double* rel,
                   cudaStream_t s);
void bks_offset_copy(const int32_t* src, int64_t count, int32_t add, int32_t* dst, cudaStream_t s);
}  // namespace fe
