// One Lanczos step on the device: KrylovSubspace::build_one
// (src/core/KrylovSubspace.cpp:125-131) for a standard problem, with every scalar kept
// in device memory so a caller can queue steps back to back (and capture them in a
// CUDA graph) without a host round trip per step.
//
//   beta      = *fnorm                         (||f|| of the previous step)
//   V[:, j]   = f / beta                       normalize_residual_into_basis (:133-147)
//   w         = A V[:, j]                      apply_operator_to_basis_column (:149-154)
//   h  = V_j^T w, w -= V_j h                   orthogonalize_active_columns, two passes
//   h2 = V_j^T w, w -= V_j h2                  over V_j = V[:, 0..j] (:156-159)
//   alpha     = h[j] + h2[j]
//   f         = w, *fnorm = ||f||              residual_norm (:161-178)
//   T[j, j]   = alpha, T[j, j-1] = T[j-1, j] = beta (j > 0)
//                                              (src/gpu/CudaLanczosKernels.cu:11-22)
#include <algorithm>
#include <string>

#include "device.hpp"
#include "fe_common.cuh"

namespace fe {
namespace {

__global__ void lanczos_record_kernel(double* T, int64_t ldt, int64_t j, const double* beta,
                                      const double* h, const double* h2) {
  T[j + j * ldt] = h[j] + h2[j];
  if (j > 0) {
    T[j + (j - 1) * ldt] = *beta;
    T[(j - 1) + j * ldt] = *beta;
  }
}

constexpr size_t kAlign = 256;
inline size_t up(size_t b) { return (b + kAlign - 1) / kAlign * kAlign; }

struct LanczosWs {
  double *w, *h, *h2, *beta;
  void *gws, *rws;
  size_t gbytes, rbytes, total;
  LanczosWs(void* base, int64_t n, int64_t m) {
    gbytes = std::max<size_t>(gram_workspace_bytes(n, m, 1), 64);
    rbytes = std::max<size_t>(residual_workspace_bytes(n, 1), 64);
    char* p = static_cast<char*>(base);
    size_t off = 0;
    auto take = [&](size_t b) {
      char* q = p ? p + off : nullptr;
      off += up(b);
      return q;
    };
    w = reinterpret_cast<double*>(take(static_cast<size_t>(n) * sizeof(double)));
    h = reinterpret_cast<double*>(take(static_cast<size_t>(m) * sizeof(double)));
    h2 = reinterpret_cast<double*>(take(static_cast<size_t>(m) * sizeof(double)));
    beta = reinterpret_cast<double*>(take(sizeof(double)));
    gws = take(gbytes);
    rws = take(rbytes);
    total = off;
  }
};

}  // namespace
}  // namespace fe

extern "C" size_t fe_lanczos_workspace_bytes(int64_t n, int64_t m) {
  if (n <= 0 || m <= 0) return 0;
  return fe::LanczosWs(nullptr, n, m).total;
}

extern "C" int fe_lanczos_step(fe_csr_t A, double* V, int64_t ldv, int64_t m, int64_t j, double* f,
                               double* fnorm, double* T, int64_t ldt, void* workspace,
                               size_t workspace_bytes, void* stream) {
  return fe::guarded("fe_lanczos_step", [&] {
    FE_REQUIRE(A, "null CSR handle");
    const fe::Csr& H = A->m;
    const int64_t n = H.rows;
    FE_REQUIRE(H.rows == H.cols, "fe_lanczos_step: operator must be square");
    FE_REQUIRE(m >= 1 && j >= 0 && j < m, "fe_lanczos_step: column j must be in [0, m)");
    FE_REQUIRE(V && f && fnorm && T, "fe_lanczos_step: null pointer");
    FE_REQUIRE(ldv >= m, "fe_lanczos_step: ldv < m");
    FE_REQUIRE(ldt >= m, "fe_lanczos_step: ldt < m");
    fe::LanczosWs ws(workspace, n, m);
    FE_REQUIRE(workspace && workspace_bytes >= ws.total,
               "fe_lanczos_step: workspace too small (need " + std::to_string(ws.total) + " bytes)");
    cudaStream_t s = fe::as_stream(stream);
    const int64_t k = j + 1;
    // beta of this step (kept for the T entries; fnorm is overwritten below).
    FE_CHECK_CUDA(cudaMemcpyAsync(ws.beta, fnorm, sizeof(double), cudaMemcpyDeviceToDevice, s));
    fe::scale_by_inv(n, f, fnorm, V + j, ldv, s);
    fe::csr_spmm<double>(H, V + j, ldv, ws.w, 1, nullptr, 0, 1, 1.0, 0.0, 0.0, s);
    fe::gram<double>(V, ldv, ws.w, 1, n, k, 1, ws.h, k, ws.gws, ws.gbytes, s);
    fe::rotate<double>(V, ldv, ws.h, k, ws.w, 1, n, k, 1, -1.0, 1.0, s);
    fe::gram<double>(V, ldv, ws.w, 1, n, k, 1, ws.h2, k, ws.gws, ws.gbytes, s);
    fe::rotate<double>(V, ldv, ws.h2, k, ws.w, 1, n, k, 1, -1.0, 1.0, s);
    fe::vec_axpby(n, 1.0, ws.w, 1, 0.0, f, 1, s);
    fe::residual_norms<double>(nullptr, f, nullptr, 1, n, 1, nullptr, nullptr, 0, nullptr, fnorm,
                               nullptr, ws.rws, ws.rbytes, s, 0);
    fe::lanczos_record_kernel<<<1, 1, 0, s>>>(T, ldt, j, ws.beta, ws.h, ws.h2);
    fe::check_launch("lanczos_record_kernel");
  });
}
