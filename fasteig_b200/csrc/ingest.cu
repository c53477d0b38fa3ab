// CSR ingestion on the device: triplets (COO, 0-based) -> the full-storage CSR
// that fasteig builds on the host with Eigen:
//   build_sparse_matrix_from_triplets (src/fasteig_problem.cpp:474-506): duplicates
//     summed left to right in input order (Eigen's setFromTriplets with a + b);
//   build_csr_from_sparse_matrix (src/fasteig_problem.cpp:554-607): every stored
//     off-diagonal (r, c, v) also contributes (c, r, v) (or -v, skew), positions that
//     receive two contributions hold their sum, rows sorted by column, explicit
//     zeros kept.
// The merged matrix holds at most one entry per position, so the second stage sums
// at most two values per position and its order does not change the result; the
// first stage keeps input order by sorting each row's entries on (column, input
// index) before the left-to-right sums. Everything after the upload runs on the
// device: a row histogram, a prefix scan, a scatter into row buckets, and one thread
// per row for the in-row sort and merge (rows of sparse operators are short).
// MatrixMarket coordinate files are parsed on the host into triplets
// (src/mmio.cpp: banner, size line, 1-based entries) and take the same path.
#include <algorithm>
#include <cctype>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "device.hpp"
#include "fe_common.cuh"

namespace fe {

namespace {

constexpr int kThreads = 256;

inline unsigned grid_for(int64_t n) {
  return static_cast<unsigned>(std::min<int64_t>(std::max<int64_t>((n + kThreads - 1) / kThreads, 1),
                                                 int64_t(148) * 64));
}

// Device buffer owned by one ingestion call.
template <typename T>
struct Tmp {
  T* p = nullptr;
  explicit Tmp(int64_t count) {
    FE_CHECK_CUDA(cudaMalloc(&p, static_cast<size_t>(std::max<int64_t>(count, 1)) * sizeof(T)));
  }
  ~Tmp() { cudaFree(p); }
  Tmp(const Tmp&) = delete;
  Tmp& operator=(const Tmp&) = delete;
};

__global__ void check_and_count_kernel(int64_t n, int64_t count, const int32_t* __restrict__ r,
                                       const int32_t* __restrict__ c, int32_t* __restrict__ cnt,
                                       int32_t* __restrict__ bad) {
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < count;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t i = r[e], j = c[e];
    if (i < 0 || j < 0 || i >= n || j >= n) {
      atomicExch(bad, 1);
      continue;
    }
    atomicAdd(&cnt[i], 1);
  }
}

// Exclusive scan in blocks of 1024: per-block scan, block totals to `sums`.
// Items at or past n_in read as zero; out gets n_out items.
template <typename T>
__global__ void scan_block_kernel(const T* __restrict__ in, int64_t n_in, int64_t n_out,
                                  int64_t* __restrict__ out, int64_t* __restrict__ sums) {
  __shared__ int64_t warp_tot[32];
  const int64_t i = static_cast<int64_t>(blockIdx.x) * 1024 + threadIdx.x;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t v = i < n_in ? static_cast<int64_t>(in[i]) : 0;
  int64_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[w] = x;
  __syncthreads();
  if (w == 0) {
    int64_t t = warp_tot[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    warp_tot[lane] = t;
  }
  __syncthreads();
  const int64_t base = w > 0 ? warp_tot[w - 1] : 0;
  if (i < n_out) out[i] = base + x - v;
  if (threadIdx.x == 1023) sums[blockIdx.x] = base + x;
}

__global__ void scan_add_kernel(int64_t* __restrict__ out, int64_t n,
                                const int64_t* __restrict__ offs) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * 1024 + threadIdx.x;
  if (i < n) out[i] += offs[blockIdx.x];
}

__global__ void narrow_kernel(const int64_t* __restrict__ in, int64_t n, int32_t* __restrict__ out) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] = static_cast<int32_t>(in[i]);
}

__global__ void row_max_kernel(int64_t n, const int64_t* __restrict__ rp, int* __restrict__ mx) {
  int local = 0;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    local = max(local, static_cast<int>(rp[i + 1] - rp[i]));
  for (int o = 16; o > 0; o >>= 1) local = max(local, __shfl_xor_sync(0xffffffffu, local, o));
  if ((threadIdx.x & 31) == 0) atomicMax(mx, local);
}

// Exclusive scan of n items: out[i] = in[0] + ... + in[i-1] for i <= n (out[n] is
// the total). Block totals are scanned by the same kernels, recursively.
template <typename T>
void exclusive_scan(const T* in, int64_t n, int64_t* out, cudaStream_t s) {
  const int64_t items = n + 1;  // item n reads as zero
  const int64_t blocks = (items + 1023) / 1024;
  Tmp<int64_t> sums(blocks);
  scan_block_kernel<T><<<static_cast<unsigned>(blocks), 1024, 0, s>>>(in, n, items, out, sums.p);
  check_launch("scan_block_kernel");
  if (blocks > 1) {
    Tmp<int64_t> offs(blocks + 1);
    exclusive_scan<int64_t>(sums.p, blocks, offs.p, s);
      scan_add_kernel<<<static_cast<unsigned>(blocks), 1024, 0, s>>>(out, items, offs.p);
    check_launch("scan_add_kernel");
    FE_CHECK_CUDA(cudaStreamSynchronize(s));  // before `offs` is freed
  }
  FE_CHECK_CUDA(cudaStreamSynchronize(s));  // before `sums` is freed
}

// Scatter entry e into its row bucket (arbitrary slot order; the in-row sort
// restores (column, input index) order).
__global__ void scatter_kernel(int64_t count, const int32_t* __restrict__ r,
                               const int32_t* __restrict__ c, const int64_t* __restrict__ start,
                               int32_t* __restrict__ fill, int32_t* __restrict__ bcol,
                               int64_t* __restrict__ bidx) {
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < count;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t i = r[e];
    const int64_t p = start[i] + atomicAdd(&fill[i], 1);
    bcol[p] = c[e];
    bidx[p] = e;
  }
}

// One thread per row: insertion sort of the row's bucket on (column, input index),
// then left-to-right sums of equal columns. Writes the merged row in place
// (mcol/mval at the bucket's start) and its length to mcnt.
__global__ void sort_merge_kernel(int64_t n, const int64_t* __restrict__ start,
                                  int32_t* __restrict__ bcol, int64_t* __restrict__ bidx,
                                  const double* __restrict__ val, double* __restrict__ mval,
                                  int32_t* __restrict__ mcnt) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t b = start[i], e = start[i + 1];
    for (int64_t p = b + 1; p < e; ++p) {
      const int32_t kc = bcol[p];
      const int64_t ki = bidx[p];
      int64_t q = p - 1;
      while (q >= b && (bcol[q] > kc || (bcol[q] == kc && bidx[q] > ki))) {
        bcol[q + 1] = bcol[q];
        bidx[q + 1] = bidx[q];
        --q;
      }
      bcol[q + 1] = kc;
      bidx[q + 1] = ki;
    }
    int64_t out = b;
    for (int64_t p = b; p < e;) {
      const int32_t col = bcol[p];
      double acc = val[bidx[p]];
      int64_t q = p + 1;
      for (; q < e && bcol[q] == col; ++q) acc = acc + val[bidx[q]];
      bcol[out] = col;
      mval[out] = acc;
      ++out;
      p = q;
    }
    mcnt[i] = static_cast<int32_t>(out - b);
  }
}

// Mirrored contributions per row: count the off-diagonal merged entries whose
// column is the row.
__global__ void mirror_count_kernel(int64_t n, const int64_t* __restrict__ start,
                                    const int32_t* __restrict__ mcnt,
                                    const int32_t* __restrict__ mcol, int32_t* __restrict__ cnt) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t b = start[i];
    for (int32_t t = 0; t < mcnt[i]; ++t) {
      const int32_t c = mcol[b + t];
      if (c != i) atomicAdd(&cnt[c], 1);
    }
  }
}

__global__ void add_counts_kernel(int64_t n, const int32_t* __restrict__ a,
                                  int32_t* __restrict__ b) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    b[i] += a[i];
}

// Row i's own merged entries go to the front of its expanded bucket (in column
// order); the mirrored entries (c -> i) follow in any order.
__global__ void expand_scatter_kernel(int64_t n, const int64_t* __restrict__ start,
                                      const int32_t* __restrict__ mcnt,
                                      const int32_t* __restrict__ mcol,
                                      const double* __restrict__ mval,
                                      const int64_t* __restrict__ fstart,
                                      int32_t* __restrict__ mfill, double sign,
                                      int32_t* __restrict__ fcol, double* __restrict__ fval) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t b = start[i];
    const int64_t fb = fstart[i];
    for (int32_t t = 0; t < mcnt[i]; ++t) {
      const int32_t c = mcol[b + t];
      const double v = mval[b + t];
      fcol[fb + t] = c;
      fval[fb + t] = v;
      if (c != i) {
        const int64_t p = fstart[c] + mcnt[c] + atomicAdd(&mfill[c], 1);
        fcol[p] = static_cast<int32_t>(i);
        fval[p] = sign * v;
      }
    }
  }
}

// One thread per row of the expanded buckets: sort on column (a position holds
// at most its own entry and one mirrored entry, whose sum is order-free) and merge.
__global__ void expand_merge_kernel(int64_t n, const int64_t* __restrict__ fstart,
                                    int32_t* __restrict__ fcol, double* __restrict__ fval,
                                    int32_t* __restrict__ fcnt) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t b = fstart[i], e = fstart[i + 1];
    for (int64_t p = b + 1; p < e; ++p) {
      const int32_t kc = fcol[p];
      const double kv = fval[p];
      int64_t q = p - 1;
      while (q >= b && fcol[q] > kc) {
        fcol[q + 1] = fcol[q];
        fval[q + 1] = fval[q];
        --q;
      }
      fcol[q + 1] = kc;
      fval[q + 1] = kv;
    }
    int64_t out = b;
    for (int64_t p = b; p < e;) {
      const int32_t col = fcol[p];
      double acc = fval[p];
      int64_t q = p + 1;
      for (; q < e && fcol[q] == col; ++q) acc = acc + fval[q];
      fcol[out] = col;
      fval[out] = acc;
      ++out;
      p = q;
    }
    fcnt[i] = static_cast<int32_t>(out - b);
  }
}

// Copy each row's merged prefix [start[i], start[i] + cnt[i]) to the final CSR
// position rowptr[i].
__global__ void compact_kernel(int64_t n, const int64_t* __restrict__ start,
                               const int32_t* __restrict__ cnt, const int64_t* __restrict__ rowptr,
                               const int32_t* __restrict__ col, const double* __restrict__ val,
                               int32_t* __restrict__ ocol, double* __restrict__ oval) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t b = start[i], o = rowptr[i];
    for (int32_t t = 0; t < cnt[i]; ++t) {
      ocol[o + t] = col[b + t];
      oval[o + t] = val[b + t];
    }
  }
}

}  // namespace

// Device build of the full-storage CSR from host triplets; the result is a
// handle like fe_csr_create's (FP64 and FP32 values on the device).
Csr* csr_from_triplets(int64_t n, int64_t count, const int32_t* rows, const int32_t* cols,
                       const double* vals, int expand) {
  // build_sparse_matrix_from_triplets's checks (src/fasteig_problem.cpp:480-497)
  FE_REQUIRE(n > 0, "Invalid matrix dimension n <= 0.");
  FE_REQUIRE(count >= 0, "Invalid nnz < 0.");
  FE_REQUIRE(n < 0x7fffffffLL, "CSR conversion requires int-sized dimensions.");
  FE_REQUIRE(count == 0 || (rows && cols && vals), "Triplet arrays inconsistent with nnz.");
  FE_REQUIRE(expand >= 0 && expand <= 2, "expand must be 0 (none), 1 (symmetric) or 2 (skew)");
  cudaStream_t s = nullptr;
  Tmp<int32_t> r(count), c(count), cnt(n), bad(1), fill(n);
  Tmp<double> v(count);
  if (count > 0) {
    FE_CHECK_CUDA(cudaMemcpy(r.p, rows, count * sizeof(int32_t), cudaMemcpyHostToDevice));
    FE_CHECK_CUDA(cudaMemcpy(c.p, cols, count * sizeof(int32_t), cudaMemcpyHostToDevice));
    FE_CHECK_CUDA(cudaMemcpy(v.p, vals, count * sizeof(double), cudaMemcpyHostToDevice));
  }
  FE_CHECK_CUDA(cudaMemsetAsync(cnt.p, 0, n * sizeof(int32_t), s));
  FE_CHECK_CUDA(cudaMemsetAsync(fill.p, 0, n * sizeof(int32_t), s));
  FE_CHECK_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int32_t), s));
  check_and_count_kernel<<<grid_for(count), kThreads, 0, s>>>(n, count, r.p, c.p, cnt.p, bad.p);
  check_launch("check_and_count_kernel");
  int32_t bad_h = 0;
  FE_CHECK_CUDA(cudaMemcpy(&bad_h, bad.p, sizeof(int32_t), cudaMemcpyDeviceToHost));
  FE_REQUIRE(bad_h == 0, "Triplet index out of bounds.");

  // Stage 1: merge duplicates in input order.
  Tmp<int64_t> start(n + 1);
  exclusive_scan(cnt.p, n, start.p, s);
  Tmp<int32_t> bcol(count), mcnt(n);
  Tmp<int64_t> bidx(count);
  Tmp<double> mval(count);
  scatter_kernel<<<grid_for(count), kThreads, 0, s>>>(count, r.p, c.p, start.p, fill.p, bcol.p,
                                                      bidx.p);
  check_launch("scatter_kernel");
  sort_merge_kernel<<<grid_for(n), kThreads, 0, s>>>(n, start.p, bcol.p, bidx.p, v.p, mval.p,
                                                     mcnt.p);
  check_launch("sort_merge_kernel");

  const int32_t* fin_cnt = mcnt.p;
  const int64_t* fin_start = start.p;
  const int32_t* fin_col = bcol.p;
  const double* fin_val = mval.p;
  // Stage 2: symmetric (or skew) expansion of the merged matrix.
  int64_t total_m = 0;
  FE_CHECK_CUDA(cudaMemcpy(&total_m, start.p + n, sizeof(int64_t), cudaMemcpyDeviceToHost));
  Tmp<int32_t> ecnt(expand ? n : 1), efill(expand ? n : 1), fcnt(expand ? n : 1);
  Tmp<int64_t> fstart(expand ? n + 1 : 1);
  Tmp<int32_t> fcol(expand ? 2 * total_m : 1);
  Tmp<double> fval(expand ? 2 * total_m : 1);
  if (expand) {
    FE_CHECK_CUDA(cudaMemsetAsync(ecnt.p, 0, n * sizeof(int32_t), s));
    FE_CHECK_CUDA(cudaMemsetAsync(efill.p, 0, n * sizeof(int32_t), s));
      mirror_count_kernel<<<grid_for(n), kThreads, 0, s>>>(n, start.p, mcnt.p, bcol.p, ecnt.p);
    check_launch("mirror_count_kernel");
      add_counts_kernel<<<grid_for(n), kThreads, 0, s>>>(n, mcnt.p, ecnt.p);
    check_launch("add_counts_kernel");
    exclusive_scan(ecnt.p, n, fstart.p, s);
      expand_scatter_kernel<<<grid_for(n), kThreads, 0, s>>>(n, start.p, mcnt.p, bcol.p, mval.p,
                                                           fstart.p, efill.p,
                                                           expand == 2 ? -1.0 : 1.0, fcol.p,
                                                           fval.p);
    check_launch("expand_scatter_kernel");
      expand_merge_kernel<<<grid_for(n), kThreads, 0, s>>>(n, fstart.p, fcol.p, fval.p, fcnt.p);
    check_launch("expand_merge_kernel");
    fin_cnt = fcnt.p;
    fin_start = fstart.p;
    fin_col = fcol.p;
    fin_val = fval.p;
  }
  // Final CSR: rowptr = scan of the merged row lengths; compact the rows into the
  // handle's own arrays (the FP32 value copy is rounded on the device).
  Tmp<int64_t> rp64(n + 1);
  exclusive_scan(fin_cnt, n, rp64.p, s);
  int64_t nnz = 0;
  FE_CHECK_CUDA(cudaMemcpy(&nnz, rp64.p + n, sizeof(int64_t), cudaMemcpyDeviceToHost));
  FE_REQUIRE(nnz <= 0x7fffffffLL, "CSR conversion produced too many nonzeros for int indexing.");
  auto* A = new Csr();
  A->rows = A->cols = n;
  A->nnz = nnz;
  FE_CHECK_CUDA(cudaGetDevice(&A->device));
  try {
    FE_CHECK_CUDA(cudaMalloc(&A->rowptr, (n + 1) * sizeof(int32_t)));
    FE_CHECK_CUDA(cudaMalloc(&A->colind, std::max<int64_t>(nnz, 1) * sizeof(int32_t)));
    FE_CHECK_CUDA(cudaMalloc(&A->val64, std::max<int64_t>(nnz, 1) * sizeof(double)));
    FE_CHECK_CUDA(cudaMalloc(&A->val32, std::max<int64_t>(nnz, 1) * sizeof(float)));
      compact_kernel<<<grid_for(n), kThreads, 0, s>>>(n, fin_start, fin_cnt, rp64.p, fin_col,
                                                    fin_val, A->colind, A->val64);
    check_launch("compact_kernel");
      narrow_kernel<<<grid_for(n + 1), kThreads, 0, s>>>(rp64.p, n + 1, A->rowptr);
    check_launch("narrow_kernel");
    if (nnz > 0) convert<double, float>(A->val64, 1, A->val32, 1, nnz, 1, s);
    Tmp<int> mx(1);
    FE_CHECK_CUDA(cudaMemsetAsync(mx.p, 0, sizeof(int), s));
      row_max_kernel<<<grid_for(n), kThreads, 0, s>>>(n, rp64.p, mx.p);
    check_launch("row_max_kernel");
    int mx_h = 0;
    FE_CHECK_CUDA(cudaMemcpyAsync(&mx_h, mx.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    FE_CHECK_CUDA(cudaStreamSynchronize(s));
    A->max_row_nnz = mx_h;
  } catch (...) {
    cudaFree(A->rowptr);
    cudaFree(A->colind);
    cudaFree(A->val64);
    cudaFree(A->val32);
    delete A;
    throw;
  }
  return A;
}

// MatrixMarket coordinate reader (src/mmio.cpp): banner "%%MatrixMarket matrix
// coordinate <real|integer|pattern> <general|symmetric|skew-symmetric>", comment
// lines, "rows cols entries", then 1-based "i j [value]" lines.
void read_matrix_market(const std::string& path, int64_t& n, std::vector<int32_t>& rows,
                        std::vector<int32_t>& cols, std::vector<double>& vals, int& expand) {
  std::ifstream in(path);
  FE_REQUIRE(in.good(), "cannot open MatrixMarket file: " + path);
  std::string line;
  FE_REQUIRE(static_cast<bool>(std::getline(in, line)), "empty MatrixMarket file: " + path);
  std::string lw = line;
  for (auto& ch : lw) ch = static_cast<char>(std::tolower(static_cast<unsigned char>(ch)));
  std::istringstream b(lw);
  std::string tag, object, format, field, sym;
  b >> tag >> object >> format >> field >> sym;
  FE_REQUIRE(tag == "%%matrixmarket" && object == "matrix" && format == "coordinate",
             "unsupported MatrixMarket banner: " + line);
  FE_REQUIRE(field == "real" || field == "integer" || field == "pattern",
             "unsupported MatrixMarket field: " + field);
  FE_REQUIRE(sym == "general" || sym == "symmetric" || sym == "skew-symmetric",
             "unsupported MatrixMarket symmetry: " + sym);
  expand = sym == "symmetric" ? 1 : (sym == "skew-symmetric" ? 2 : 0);
  while (std::getline(in, line)) {
    if (!line.empty() && line[0] != '%') break;
  }
  long long nr = 0, nc = 0, nz = 0;
  {
    std::istringstream sz(line);
    FE_REQUIRE(static_cast<bool>(sz >> nr >> nc >> nz), "invalid MatrixMarket size line");
  }
  FE_REQUIRE(nr == nc, "CSR conversion requires a square matrix.");
  n = nr;
  rows.resize(static_cast<size_t>(nz));
  cols.resize(static_cast<size_t>(nz));
  vals.resize(static_cast<size_t>(nz));
  for (long long e = 0; e < nz; ++e) {
    long long i = 0, j = 0;
    double v = 1.0;
    FE_REQUIRE(static_cast<bool>(in >> i >> j), "truncated MatrixMarket entries");
    if (field != "pattern") FE_REQUIRE(static_cast<bool>(in >> v), "truncated MatrixMarket entries");
    rows[static_cast<size_t>(e)] = static_cast<int32_t>(i - 1);
    cols[static_cast<size_t>(e)] = static_cast<int32_t>(j - 1);
    vals[static_cast<size_t>(e)] = v;
  }
}

}  // namespace fe

extern "C" int fe_csr_create_from_triplets(int64_t n, int64_t count, const int32_t* rows,
                                           const int32_t* cols, const double* values,
                                           int32_t expand, fe_csr_t* out) {
  return fe::guarded("fe_csr_create_from_triplets", [&] {
    FE_REQUIRE(out, "null output handle");
    *out = nullptr;
    fe::Csr* A = fe::csr_from_triplets(n, count, rows, cols, values, expand);
    auto* h = new fe_csr();
    h->m = *A;
    delete A;
    *out = h;
  });
}

extern "C" int fe_csr_create_from_matrix_market(const char* path, fe_csr_t* out) {
  return fe::guarded("fe_csr_create_from_matrix_market", [&] {
    FE_REQUIRE(path && out, "null argument");
    *out = nullptr;
    int64_t n = 0;
    int expand = 0;
    std::vector<int32_t> r, c;
    std::vector<double> v;
    fe::read_matrix_market(path, n, r, c, v, expand);
    fe::Csr* A = fe::csr_from_triplets(n, static_cast<int64_t>(v.size()), r.data(), c.data(),
                                       v.data(), expand);
    auto* h = new fe_csr();
    h->m = *A;
    delete A;
    *out = h;
  });
}
