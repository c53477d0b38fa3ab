// Kernels of the grouped Chebyshev engine (grouped.cpp): assembly of the
// concatenated block-diagonal operator, its per-member filter scaling, the
// per-member reduction of Gram partials, and per-member residual norms.
//
// Layout: member p owns rows [row0_p, row0_p + n_pad_p) of every concatenated
// block (row-major, one common width), n_pad_p a multiple of the 128-row rotation
// tile, the rows past its n_p empty in the operator and zero in every block. A
// row tile, and every Gram chunk, lies inside one member, so each member's
// products read only its own rows and sum them in the same order whatever else is
// in the group.

#include "grouped.hpp"

namespace fe {
namespace {

constexpr int kPackThreads = 256;

unsigned grid_for(int64_t count, int per_block) {
  const int64_t blocks = (count + per_block - 1) / per_block;
  return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(blocks, 148 * 16)));
}

__global__ void pack_rowptr_kernel(const int32_t* __restrict__ rowptr, int64_t n, int64_t n_pad,
                                   int64_t nz0, int32_t* __restrict__ out) {
  const int32_t base = rowptr[0];
  const int32_t last = rowptr[n];
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n_pad;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t v = i < n ? rowptr[i] : last;
    out[i] = static_cast<int32_t>(nz0 + (v - base));
  }
}

__global__ void pack_entries_kernel(const int32_t* __restrict__ colind,
                                    const double* __restrict__ val, int64_t nnz, int32_t col_add,
                                    double sign, int32_t* __restrict__ cat_colind,
                                    double* __restrict__ cat_plain) {
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < nnz;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    cat_colind[j] = colind[j] + col_add;
    cat_plain[j] = sign * val[j];
  }
}

__global__ void bad_diagonal_kernel(const int32_t* __restrict__ rowptr,
                                    const int32_t* __restrict__ colind, int64_t n,
                                    int32_t* __restrict__ count) {
  int32_t bad = 0;
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int hits = 0;
    for (int32_t j = rowptr[r]; j < rowptr[r + 1]; ++j) hits += colind[j] == r;
    bad += hits != 1;
  }
  if (bad) atomicAdd(count, bad);
}

// One thread per row: the scaled operator c A + d I of the row's member (the
// reference's filter operator, src/ChebyshevSolver.cpp:231-245).
template <typename T>
__global__ void rescale_kernel(const int32_t* __restrict__ rowptr,
                               const int32_t* __restrict__ colind,
                               const double* __restrict__ plain, T* __restrict__ scaled,
                               int64_t rows, const int32_t* __restrict__ tile_member,
                               const double* __restrict__ cd) {
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < rows;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int p = tile_member[r / kRotateRowTile];
    const double c = cd[2 * p];
    const double d = cd[2 * p + 1];
    for (int32_t j = rowptr[r]; j < rowptr[r + 1]; ++j)
      scaled[j] = static_cast<T>(c * plain[j] + (colind[j] == r ? d : 0.0));
  }
}

// Gram partials of gram_dmma_kernel are [chunk][j][i] (column-major k x m per
// chunk); with `symmetric` only the 64 x 64 tiles on and above the diagonal hold
// data and the rest read their mirror.
__global__ void gram_reduce_members_kernel(const double* __restrict__ partial, int k, int m,
                                           const int32_t* __restrict__ member_chunks,
                                           int symmetric, double* __restrict__ G,
                                           int64_t stride) {
  const int p = blockIdx.y;
  const int64_t idx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t total = static_cast<int64_t>(k) * m;
  if (idx >= total) return;
  const int i = static_cast<int>(idx % k);
  const int j = static_cast<int>(idx / k);
  const int64_t src = (symmetric && i / 64 > j / 64) ? static_cast<int64_t>(i) * k + j : idx;
  const int c0 = member_chunks[2 * p];
  const int nc = member_chunks[2 * p + 1];
  double s = 0.0;
  for (int c = c0; c < c0 + nc; ++c) s += partial[static_cast<int64_t>(c) * total + src];
  G[static_cast<int64_t>(p) * stride + static_cast<int64_t>(j) * k + i] = s;
}

// One CTA per chunk (rows of one member): thread t takes column t % width (of a
// 256-column slice) and every (256 / width)-th row, then the row lanes are added in
// lane order through shared memory. Sums of (AX - theta X)^2 and X^2 per column.
constexpr int kResidThreads = 256;

__global__ void __launch_bounds__(kResidThreads)
resid_partial_kernel(const double* __restrict__ AX, const double* __restrict__ X, int64_t ld,
                     int width, const int64_t* __restrict__ chunk_rows,
                     const int32_t* __restrict__ chunk_member, const double* __restrict__ theta,
                     double* __restrict__ partial) {
  __shared__ double red[2][kResidThreads];
  const int c = blockIdx.x;
  const int p = chunk_member[c];
  const int64_t r0 = chunk_rows[2 * c];
  const int64_t r1 = chunk_rows[2 * c + 1];
  const int slice = min(width, kResidThreads);
  const int lanes = kResidThreads / slice;
  const int col = threadIdx.x % slice;
  const int lane = threadIdx.x / slice;
  for (int j0 = 0; j0 < width; j0 += slice) {
    const int j = j0 + col;
    double rs = 0.0, xs = 0.0;
    if (lane < lanes && j < width) {
      const double th = theta[static_cast<int64_t>(p) * width + j];
#pragma unroll 4
      for (int64_t r = r0 + lane; r < r1; r += lanes) {
        const double x = X[r * ld + j];
        const double d = AX[r * ld + j] - th * x;
        rs = fma(d, d, rs);
        xs = fma(x, x, xs);
      }
    }
    red[0][threadIdx.x] = rs;
    red[1][threadIdx.x] = xs;
    __syncthreads();
    if (lane == 0 && j < width) {
      for (int l = 1; l < lanes; ++l) {
        rs += red[0][l * slice + col];
        xs += red[1][l * slice + col];
      }
      partial[static_cast<int64_t>(c) * 2 * width + j] = rs;
      partial[static_cast<int64_t>(c) * 2 * width + width + j] = xs;
    }
    __syncthreads();
  }
}

// The reference's relative residual (src/core/RitzExtraction.cpp:127-140).
__global__ void resid_finish_kernel(const double* __restrict__ partial, int width,
                                    const int32_t* __restrict__ member_chunks,
                                    const double* __restrict__ theta, double* __restrict__ rel) {
  const int p = blockIdx.x;
  const int c0 = member_chunks[2 * p];
  const int nc = member_chunks[2 * p + 1];
  for (int j = threadIdx.x; j < width; j += blockDim.x) {
    double rs = 0.0, xs = 0.0;
    for (int c = c0; c < c0 + nc; ++c) {
      rs += partial[static_cast<int64_t>(c) * 2 * width + j];
      xs += partial[static_cast<int64_t>(c) * 2 * width + width + j];
    }
    const double th = theta[static_cast<int64_t>(p) * width + j];
    const double den = (1.0 + fabs(th)) * sqrt(xs);
    rel[static_cast<int64_t>(p) * width + j] = den > 0.0 ? sqrt(rs) / den : sqrt(rs);
  }
}

}  // namespace

void group_pack_member(const Csr& A, int64_t row0, int64_t n_pad, int64_t nz0, double sign,
                       int32_t* cat_rowptr, int32_t* cat_colind, double* cat_plain,
                       cudaStream_t s) {
  FE_REQUIRE(A.val64 != nullptr, "grouped Chebyshev: operator has no FP64 values");
  FE_REQUIRE(n_pad >= A.rows && n_pad % kRotateRowTile == 0, "grouped pack: bad row padding");
  pack_rowptr_kernel<<<grid_for(n_pad, kPackThreads), kPackThreads, 0, s>>>(
      A.rowptr, A.rows, n_pad, nz0, cat_rowptr + row0);
  check_launch("pack_rowptr_kernel");
  if (A.nnz > 0) {
    pack_entries_kernel<<<grid_for(A.nnz, kPackThreads), kPackThreads, 0, s>>>(
        A.colind, A.val64, A.nnz, static_cast<int32_t>(row0), sign, cat_colind + nz0,
        cat_plain + nz0);
    check_launch("pack_entries_kernel");
  }
}

void csr_count_bad_diagonals(const Csr& A, int32_t* count, cudaStream_t s) {
  FE_CHECK_CUDA(cudaMemsetAsync(count, 0, sizeof(int32_t), s));
  if (A.rows == 0) return;
  bad_diagonal_kernel<<<grid_for(A.rows, kPackThreads), kPackThreads, 0, s>>>(A.rowptr, A.colind,
                                                                              A.rows, count);
  check_launch("bad_diagonal_kernel");
}

void group_rescale(const int32_t* rowptr, const int32_t* colind, const double* plain,
                   double* scaled, int64_t rows, const int32_t* tile_member, const double* cd,
                   cudaStream_t s) {
  if (rows == 0) return;
  rescale_kernel<double><<<grid_for(rows, kPackThreads), kPackThreads, 0, s>>>(
      rowptr, colind, plain, scaled, rows, tile_member, cd);
  check_launch("rescale_kernel");
}

void group_rescale_f32(const int32_t* rowptr, const int32_t* colind, const double* plain,
                       float* scaled, int64_t rows, const int32_t* tile_member, const double* cd,
                       cudaStream_t s) {
  if (rows == 0) return;
  rescale_kernel<float><<<grid_for(rows, kPackThreads), kPackThreads, 0, s>>>(
      rowptr, colind, plain, scaled, rows, tile_member, cd);
  check_launch("rescale_kernel");
}

void group_gram_reduce(const double* partial, int k, int m, int members,
                       const int32_t* member_chunks, bool symmetric, double* G, int64_t stride,
                       cudaStream_t s) {
  const int64_t total = static_cast<int64_t>(k) * m;
  FE_REQUIRE(members >= 1 && members <= 65535, "grouped Gram: member count out of range");
  dim3 grid(static_cast<unsigned>((total + 255) / 256), static_cast<unsigned>(members));
  gram_reduce_members_kernel<<<grid, 256, 0, s>>>(partial, k, m, member_chunks,
                                                  symmetric ? 1 : 0, G, stride);
  check_launch("gram_reduce_members_kernel");
}

void group_residuals(const double* AX, const double* X, int64_t ld, int width, int chunks,
                     const int64_t* chunk_rows, const int32_t* chunk_member, int members,
                     const int32_t* member_chunks, const double* theta, double* partial,
                     double* rel, cudaStream_t s) {
  const int threads = std::min(256, (width + 31) / 32 * 32);
  resid_partial_kernel<<<static_cast<unsigned>(chunks), kResidThreads, 0, s>>>(
      AX, X, ld, width, chunk_rows, chunk_member, theta, partial);
  check_launch("resid_partial_kernel");
  resid_finish_kernel<<<static_cast<unsigned>(members), threads, 0, s>>>(partial, width,
                                                                          member_chunks, theta, rel);
  check_launch("resid_finish_kernel");
}

}  // namespace fe
