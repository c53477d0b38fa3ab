// Shared helpers for the fasteig_b200 CUDA backend (sm_100a).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

#include "../../include/fasteig_b200.h"

namespace fe {

// Thread-local message behind fe_last_error().
void set_last_error(const std::string& msg);

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define FE_CHECK_CUDA(call)                                                        \
  do {                                                                             \
    cudaError_t fe_err_ = (call);                                                  \
    if (fe_err_ != cudaSuccess) {                                                  \
      throw ::fe::Error(FE_ERR_CUDA, std::string(#call) + " failed: " +            \
                                         cudaGetErrorString(fe_err_) + " @" +      \
                                         __FILE__ + ":" + std::to_string(__LINE__)); \
    }                                                                              \
  } while (0)

#define FE_REQUIRE(cond, msg)                                   \
  do {                                                          \
    if (!(cond)) throw ::fe::Error(FE_ERR_INVALID, (msg));       \
  } while (0)

// Run `body` converting exceptions into C status codes.
template <typename F>
int guarded(const char* where, F&& body) {
  try {
    body();
    return FE_OK;
  } catch (const Error& e) {
    set_last_error(std::string(where) + ": " + e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    set_last_error(std::string(where) + ": host allocation failed");
    return FE_ERR_ALLOC;
  } catch (const std::exception& e) {
    set_last_error(std::string(where) + ": " + e.what());
    return FE_ERR_INVALID;
  }
}

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Number of this library's kernel launches since load (all threads).
void count_launch();

inline void check_launch(const char* what) {
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    throw Error(FE_ERR_CUDA, std::string(what) + " launch failed: " + cudaGetErrorString(e));
  }
}

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Do two row-major views (rows x cols, leading dimension ld) share an element?
// Views of the same buffer with equal ld and disjoint column ranges do not.
template <typename T>
inline bool ranges_overlap(const T* a, int64_t rows_a, int64_t ld_a, int64_t cols_a,
                           const T* b, int64_t rows_b, int64_t ld_b, int64_t cols_b) {
  if (rows_a <= 0 || rows_b <= 0 || cols_a <= 0 || cols_b <= 0) return false;
  const char* a0 = reinterpret_cast<const char*>(a);
  const char* a1 = reinterpret_cast<const char*>(a + (rows_a - 1) * ld_a + cols_a);
  const char* b0 = reinterpret_cast<const char*>(b);
  const char* b1 = reinterpret_cast<const char*>(b + (rows_b - 1) * ld_b + cols_b);
  if (!(a0 < b1 && b0 < a1)) return false;
  if (ld_a == ld_b && cols_a <= ld_a && cols_b <= ld_b) {
    const int64_t d = b - a;  // element offset of b relative to a
    int64_t r = d % ld_a;
    if (r < 0) r += ld_a;
    // b's columns relative to a's row grid: [r, r+cols_b), possibly wrapping.
    const bool hit = (r < cols_a) || (r + cols_b > ld_a && r + cols_b - ld_a > 0);
    return hit;
  }
  return true;
}

// Device CSR operator: int32 indices, FP64 and FP32 values.
struct Csr {
  int64_t rows = 0, cols = 0, nnz = 0;
  int32_t* rowptr = nullptr;
  int32_t* colind = nullptr;
  double* val64 = nullptr;
  float* val32 = nullptr;
  int device = 0;
  int64_t max_row_nnz = 0;
  // max |column - row| over the stored entries, measured on first use by the
  // multi-step filter (-1: not measured yet)
  mutable int64_t bandwidth = -1;
  // SpMM kernel chosen by fe_csr_autotune per precision (0 FP64, 1 FP32) for up
  // to four block widths; mode < 0 marks an empty entry.
  struct Tuned {
    int32_t ncols = 0;
    int32_t mode = -1;
  };
  Tuned tuned[2][4];
};

int num_sms();

// Device status word that kernels launched from this host thread record a
// timed-out bounded wait in: the one a solve installed for its duration
// (StatusScope), or null for the library's default word (fe_device_status).
int* current_status_word();
void set_status_word(int* word);
struct StatusScope {
  int* prev;
  explicit StatusScope(int* word) : prev(current_status_word()) { set_status_word(word); }
  ~StatusScope() { set_status_word(prev); }
  StatusScope(const StatusScope&) = delete;
  StatusScope& operator=(const StatusScope&) = delete;
};
void launch_wait_probe(int* status, long long limit_cycles, int code, cudaStream_t s);
// A status word owned by the calling host thread on the current device (allocated
// on first use and kept; solves on one thread run one at a time).
int* thread_status_word();

// FP64 tensor-core kernels (dmma.cu).
void gram_partial_dmma(const double* X, int64_t ldx, const double* Y, int64_t ldy, int64_t n,
                       int k, int m, int tiles_k, int tiles_m, int chunks, int64_t rows_per_chunk,
                       bool symmetric, double* partial, cudaStream_t s);
void rotate_dmma(const double* X, int64_t ldx, const double* C, int64_t ldc, double* Y,
                 int64_t ldy, int64_t n, int64_t k, int64_t m, double alpha, double beta,
                 cudaStream_t s, bool upper_tri = false, const int32_t* tile_member = nullptr,
                 int64_t c_stride = 0);
void gram_partial_dmma_ranges(const double* X, int64_t ldx, const double* Y, int64_t ldy, int k,
                              int m, int chunks, const int64_t* chunk_rows, bool symmetric,
                              double* partial, cudaStream_t s);
// Row tile of the FP64 rotation kernel (grouped rotations pad every problem's rows
// to a multiple of it).
constexpr int kRotateRowTile = 128;

}  // namespace fe

struct fe_csr {
  fe::Csr m;
};
