// Grouped Chebyshev engine: many standard eigenproblems advance together, one
// filter cycle at a time, over one concatenated block-diagonal operator.
//
// One cycle of every member (the reference's ChebyshevSolver loop body,
// src/ChebyshevSolver.cpp:145-205, with all columns filtered) is one launch
// sequence on the group's stream:
//   1. per-member filter operator c_p A_p + d_p I written into the scaled copy of
//      the concatenated values (c_p, d_p from the member's bounds and cutoff);
//   2. the filter recurrence Y_1 = (cA + dI) X, Y_k = 2 (cA + dI) Y_{k-1} - Y_{k-2}
//      (src/ChebyshevSolver.cpp:231-256): `degree` SpMMs over the concatenated
//      operator, every member's rows in each launch (an FP32-filter group runs them on
//      FP32 copies of X and of the scaled values and widens the result to FP64);
//   3. Cholesky QR, twice (thin_qr_in_place with QrMethod::Cholesky): grouped Gram
//      (each member's rows in its own chunks), batched Cholesky and triangular
//      inverse, grouped rotation (each row tile with its member's R^-1);
//   4. Rayleigh-Ritz (extract_projected_ritz_pairs, src/core/RitzExtraction.cpp:
//      95-141): W = A Y, grouped Gram Y^T W, batched symmetric eigensolver, the
//      grouped rotations X = Y Q and AX = W Q, and each member's relative residuals;
//   5. Ritz values, residuals and Cholesky/eigensolver status words to pinned host
//      memory.
// The host then checks each member's convergence (the first nev residuals <= tol,
// as the reference checks every cycle) and the members that finished leave. When
// members join or leave, the concatenated operator and blocks are rebuilt
// (retained members keep their current Ritz vectors); while the membership stays
// the same the sequence is captured once into a CUDA graph and replayed.

#include "grouped.hpp"

#include <cmath>
#include <cstring>
#include <limits>
#include <random>

namespace fe {
namespace {

constexpr int64_t kTile = kRotateRowTile;
constexpr int kBlocks = 5;  // 0..2 filter ring (0 holds the Ritz vectors X), 3: W = A Y, 4: A X

int64_t round_up(int64_t a, int64_t b) { return (a + b - 1) / b * b; }

// Gram / residual chunks of one member: equal row ranges (a multiple of the row
// tile, at least 2,048 rows), at most 256 of them. Depends on the member alone.
int64_t member_chunk_rows(int64_t n_pad) {
  return std::max<int64_t>(2048, round_up((n_pad + 255) / 256, kTile));
}
int64_t member_chunk_count(int64_t n_pad) {
  const int64_t r = member_chunk_rows(n_pad);
  return (n_pad + r - 1) / r;
}

struct AllocOn {
  cudaStream_t prev;
  explicit AllocOn(cudaStream_t s) : prev(alloc_stream()) { alloc_stream() = s; }
  ~AllocOn() { alloc_stream() = prev; }
};

class PinnedBuffer {
 public:
  PinnedBuffer() = default;
  ~PinnedBuffer() {
    if (p_) cudaFreeHost(p_);
  }
  PinnedBuffer(const PinnedBuffer&) = delete;
  PinnedBuffer& operator=(const PinnedBuffer&) = delete;
  void resize(size_t bytes) {
    if (bytes <= bytes_) return;
    if (p_) cudaFreeHost(p_);
    p_ = nullptr;
    bytes_ = 0;
    FE_CHECK_CUDA(cudaMallocHost(&p_, bytes));
    bytes_ = bytes;
  }
  template <typename T>
  T* as() const {
    return static_cast<T*>(p_);
  }

 private:
  void* p_ = nullptr;
  size_t bytes_ = 0;
};

// Filter scaling (src/ChebyshevSolver.cpp:231-239) of the interval [cutoff, upper];
// a collapsed interval leaves the block unfiltered (T_k(1) = 1).
void filter_scaling(double cutoff, double upper, double* c, double* d) {
  if (upper == cutoff) {
    *c = 0.0;
    *d = 1.0;
    return;
  }
  *c = 2.0 / (upper - cutoff);
  *d = -(upper + cutoff) / (upper - cutoff);
  if (!std::isfinite(*c) || !std::isfinite(*d))
    throw Error(FE_ERR_NONFINITE, "ChebyshevSolver: invalid filter scaling.");
}

}  // namespace

size_t group_member_bytes(const Csr& A, int64_t width, bool mixed) {
  const int64_t n_pad = round_up(std::max<int64_t>(A.rows, 1), kTile);
  const double blk = static_cast<double>(n_pad) * width * 8.0;
  const double csr = static_cast<double>(n_pad + 1) * 4.0 + static_cast<double>(A.nnz) * 20.0;
  const double chunks = static_cast<double>(member_chunk_count(n_pad));
  const double ws = chunks * width * width * 8.0 + chunks * 2.0 * width * 8.0 +
                    8.0 * width * width * 8.0 +
                    static_cast<double>(syevd_workspace_bytes(1, width));
  const double bounds = static_cast<double>(A.rows) * 26.0 * 8.0;  // Lanczos basis at join
  // blocks plus the new Ritz block of a repack, two operator copies during a repack;
  // mixed: three FP32 filter blocks, the FP32 operator values, the carried Ritz block
  const double extra = mixed ? 2.5 * blk + static_cast<double>(A.nnz) * 8.0 : 0.0;
  return static_cast<size_t>((kBlocks + 1) * blk + 2.0 * csr + ws + bounds + extra) +
         (size_t(16) << 20);
}

struct ChebGroup::Impl {
  int64_t R = 0, NNZ = 0, tiles = 0, chunks = 0;
  int G = 0;
  int64_t max_row_nnz = 0;
  DeviceBuffer rowptr, colind, plain, scaled, scaled32;
  DeviceBuffer blk[kBlocks];
  DeviceBuffer f32[3];  // FP32 filter ring of an FP32-filter group
  DeviceBuffer tile_member, chunk_rows, chunk_member, member_chunks;
  DeviceBuffer gpart, rpart, Gm, Rinv, Q, theta, rel, info, cd, syevd_ws;
  PinnedBuffer cd_h, theta_h, rel_h, info_h;
  Csr op_scaled, op_plain;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool dirty = true;  // membership changed since the last repack
  int eager_cycles = 0;

  void drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  }
  ~Impl() { drop_graph(); }
};

ChebGroup::ChebGroup(int device, int64_t width, int64_t degree, bool fp32_filter)
    : impl_(new Impl), device_(device), width_(width), degree_(degree), fp32_(fp32_filter) {
  FE_REQUIRE(width >= 32 && width % 32 == 0 && width <= 512, "grouped Chebyshev: invalid width");
  FE_REQUIRE(degree >= 1, "grouped Chebyshev: degree must be >= 1");
  FE_CHECK_CUDA(cudaSetDevice(device));
  retain_pool_memory(device);
  FE_CHECK_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
}

ChebGroup::~ChebGroup() {
  if (stream_) cudaStreamSynchronize(stream_);
  {
    AllocOn on(stream_);
    impl_.reset();
  }
  if (stream_) {
    cudaStreamSynchronize(stream_);
    cudaStreamDestroy(stream_);
  }
}

void ChebGroup::join(GroupMember* m) {
  FE_REQUIRE(m && m->A, "grouped Chebyshev: null member");
  FE_REQUIRE(m->g.width == width_ && m->g.degree == degree_,
             "grouped Chebyshev: member width or degree differs from the group's");
  FE_REQUIRE(!fp32_ || m->g.mixed, "grouped Chebyshev: FP64 member in an FP32-filter group");
  m->fresh = true;
  if (m->switched) {
    // from the FP32-filter group of its width: keeps its cycle count, interval and
    // Ritz block (m->carry)
    m->switched = false;
  } else {
    m->iterations = 0;
    m->fp32_iterations = 0;
    m->worst_history.clear();
    m->t_join = std::chrono::steady_clock::now();
    m->cutoff = m->g.reference_cutoff;
  }
  joining_.push_back(m);
  impl_->dirty = true;
}

void ChebGroup::fail_all(int rc, const std::string& error, std::vector<GroupMember*>& done) {
  cudaStreamSynchronize(stream_);
  cudaGetLastError();
  for (auto* list : {&members_, &joining_}) {
    for (GroupMember* m : *list) {
      m->rc = rc;
      m->error = error;
      m->switched = false;
      m->carry.release();  // while the stream it was allocated on still exists
      m->seconds =
          std::chrono::duration<double>(std::chrono::steady_clock::now() - m->t_join).count();
      done.push_back(m);
    }
    list->clear();
  }
  launched_ = false;
  impl_->drop_graph();
  impl_->dirty = true;
}

void ChebGroup::launch_cycle() {
  FE_REQUIRE(!launched_, "grouped Chebyshev: cycle already in flight");
  FE_CHECK_CUDA(cudaSetDevice(device_));
  Impl& I = *impl_;
  const int64_t b = width_;
  cudaStream_t s = stream_;
  AllocOn on(s);

  if (I.dirty) {
    // ---- repack: retained members first (their Ritz blocks carried over), then
    // the joining ones (random start blocks).
    I.drop_graph();
    std::vector<GroupMember*> order = members_;
    order.insert(order.end(), joining_.begin(), joining_.end());
    joining_.clear();
    if (order.empty()) {
      members_.clear();
      I.dirty = false;
      return;
    }
    std::vector<int64_t> old_row0(order.size(), -1);
    for (size_t p = 0; p < order.size(); ++p)
      if (!order[p]->fresh) old_row0[p] = order[p]->row0;
    int64_t R = 0, NNZ = 0, chunks = 0, maxnz = 0;
    for (GroupMember* m : order) {
      m->row0 = R;
      m->n_pad = round_up(m->A->rows, kTile);
      m->nz0 = NNZ;
      m->chunk0 = chunks;
      m->chunks = member_chunk_count(m->n_pad);
      R += m->n_pad;
      NNZ += m->A->nnz;
      chunks += m->chunks;
      maxnz = std::max(maxnz, m->A->max_row_nnz);
    }
    FE_REQUIRE(R < 0x7fffffffLL && NNZ <= 0x7fffffffLL,
               "grouped Chebyshev: concatenated operator exceeds int32 indexing");
    FE_REQUIRE(chunks <= 65535, "grouped Chebyshev: too many Gram chunks");
    const int G = static_cast<int>(order.size());
    const size_t blk_bytes = static_cast<size_t>(R) * b * sizeof(double);

    // New Ritz block: zero (padding rows stay zero), retained members copied over.
    DeviceBuffer X(blk_bytes);
    FE_CHECK_CUDA(cudaMemsetAsync(X.get(), 0, blk_bytes, s));
    for (size_t p = 0; p < order.size(); ++p) {
      if (old_row0[p] < 0) continue;
      FE_CHECK_CUDA(cudaMemcpyAsync(X.as<double>() + order[p]->row0 * b,
                                    I.blk[0].as<double>() + old_row0[p] * b,
                                    static_cast<size_t>(order[p]->n_pad) * b * sizeof(double),
                                    cudaMemcpyDeviceToDevice, s));
    }
    for (int i = 0; i < kBlocks; ++i) I.blk[i].release();
    I.rowptr.release();
    I.colind.release();
    I.plain.release();
    I.scaled.release();
    I.scaled32.release();
    for (auto& f : I.f32) f.release();
    I.gpart.release();
    I.rpart.release();

    // Start blocks of the joining members: the reference's std::mt19937 draws
    // (Executor::create_random_multivector, column-major order) or the device
    // generator, as the member's init option asks.
    for (GroupMember* m : order) {
      if (!m->fresh) continue;
      double* dst = X.as<double>() + m->row0 * b;
      if (m->carry.get()) {
        // Ritz block carried over from the FP32-filter group (same width and padding)
        FE_CHECK_CUDA(cudaMemcpyAsync(dst, m->carry.get(),
                                      static_cast<size_t>(m->n_pad) * b * sizeof(double),
                                      cudaMemcpyDeviceToDevice, s));
        continue;
      }
      if (m->g.host_init) {
        std::mt19937 rng(m->g.seed);
        std::uniform_real_distribution<double> dist(-1.0, 1.0);
        std::vector<double> host(static_cast<size_t>(m->A->rows) * b);
        for (int64_t j = 0; j < b; ++j)
          for (int64_t i = 0; i < m->A->rows; ++i)
            host[static_cast<size_t>(i) * b + j] = dist(rng);
        FE_CHECK_CUDA(cudaMemcpyAsync(dst, host.data(), host.size() * sizeof(double),
                                      cudaMemcpyHostToDevice, s));
        FE_CHECK_CUDA(cudaStreamSynchronize(s));
      } else {
        fill_uniform<double>(dst, b, m->A->rows, b, m->g.seed, s);
      }
    }
    I.blk[0] = std::move(X);
    for (int i = 1; i < kBlocks; ++i) {
      I.blk[i].resize(blk_bytes);
      FE_CHECK_CUDA(cudaMemsetAsync(I.blk[i].get(), 0, blk_bytes, s));
    }

    // Concatenated operator.
    I.rowptr.resize(static_cast<size_t>(R + 1) * sizeof(int32_t));
    I.colind.resize(static_cast<size_t>(std::max<int64_t>(NNZ, 1)) * sizeof(int32_t));
    I.plain.resize(static_cast<size_t>(std::max<int64_t>(NNZ, 1)) * sizeof(double));
    if (fp32_) {
      I.scaled32.resize(static_cast<size_t>(std::max<int64_t>(NNZ, 1)) * sizeof(float));
      for (auto& f : I.f32) {
        f.resize(static_cast<size_t>(R) * b * sizeof(float));
        FE_CHECK_CUDA(cudaMemsetAsync(f.get(), 0, static_cast<size_t>(R) * b * sizeof(float), s));
      }
    } else {
      I.scaled.resize(static_cast<size_t>(std::max<int64_t>(NNZ, 1)) * sizeof(double));
    }
    for (GroupMember* m : order)
      group_pack_member(*m->A, m->row0, m->n_pad, m->nz0, m->g.sign, I.rowptr.as<int32_t>(),
                        I.colind.as<int32_t>(), I.plain.as<double>(), s);
    {
      const int32_t last = static_cast<int32_t>(NNZ);
      FE_CHECK_CUDA(cudaMemcpyAsync(I.rowptr.as<int32_t>() + R, &last, sizeof(int32_t),
                                    cudaMemcpyHostToDevice, s));
      FE_CHECK_CUDA(cudaStreamSynchronize(s));
    }
    for (Csr* op : {&I.op_scaled, &I.op_plain}) {
      op->rows = op->cols = R;
      op->nnz = NNZ;
      op->rowptr = I.rowptr.as<int32_t>();
      op->colind = I.colind.as<int32_t>();
      op->val32 = nullptr;
      op->device = device_;
      op->max_row_nnz = maxnz;
      op->bandwidth = -1;
    }
    I.op_scaled.val64 = fp32_ ? nullptr : I.scaled.as<double>();
    I.op_scaled.val32 = fp32_ ? I.scaled32.as<float>() : nullptr;
    I.op_plain.val64 = I.plain.as<double>();

    // Tables: row tile -> member, chunk -> rows and member, member -> chunks.
    std::vector<int32_t> tile_member(R / kTile), chunk_member(chunks), member_chunks(2 * G);
    std::vector<int64_t> chunk_rows(2 * chunks);
    for (int p = 0; p < G; ++p) {
      GroupMember* m = order[p];
      for (int64_t t = m->row0 / kTile; t < (m->row0 + m->n_pad) / kTile; ++t) tile_member[t] = p;
      const int64_t rpc = member_chunk_rows(m->n_pad);
      for (int64_t c = 0; c < m->chunks; ++c) {
        chunk_rows[2 * (m->chunk0 + c)] = m->row0 + c * rpc;
        chunk_rows[2 * (m->chunk0 + c) + 1] = m->row0 + std::min(m->n_pad, (c + 1) * rpc);
        chunk_member[m->chunk0 + c] = p;
      }
      member_chunks[2 * p] = static_cast<int32_t>(m->chunk0);
      member_chunks[2 * p + 1] = static_cast<int32_t>(m->chunks);
    }
    auto upload = [&](DeviceBuffer& d, const void* h, size_t bytes) {
      d.resize(std::max<size_t>(bytes, 16));
      FE_CHECK_CUDA(cudaMemcpyAsync(d.get(), h, bytes, cudaMemcpyHostToDevice, s));
    };
    upload(I.tile_member, tile_member.data(), tile_member.size() * sizeof(int32_t));
    upload(I.chunk_member, chunk_member.data(), chunk_member.size() * sizeof(int32_t));
    upload(I.member_chunks, member_chunks.data(), member_chunks.size() * sizeof(int32_t));
    upload(I.chunk_rows, chunk_rows.data(), chunk_rows.size() * sizeof(int64_t));
    FE_CHECK_CUDA(cudaStreamSynchronize(s));  // host tables leave scope
    for (GroupMember* m : order) m->carry.release();  // copied (the stream is idle)

    // Workspaces.
    const size_t bb = static_cast<size_t>(b) * b * sizeof(double);
    I.gpart.resize(static_cast<size_t>(chunks) * bb);
    I.rpart.resize(static_cast<size_t>(chunks) * 2 * b * sizeof(double));
    I.Gm.resize(G * bb);
    I.Rinv.resize(G * bb);
    I.Q.resize(G * bb);
    I.theta.resize(static_cast<size_t>(G) * b * sizeof(double));
    I.rel.resize(static_cast<size_t>(G) * b * sizeof(double));
    I.info.resize(static_cast<size_t>(3 * G) * sizeof(int32_t));
    I.cd.resize(static_cast<size_t>(2 * G) * sizeof(double));
    I.syevd_ws.resize(syevd_workspace_bytes(G, b));
    I.cd_h.resize(static_cast<size_t>(2 * G) * sizeof(double));
    I.theta_h.resize(static_cast<size_t>(G) * b * sizeof(double));
    I.rel_h.resize(static_cast<size_t>(G) * b * sizeof(double));
    I.info_h.resize(static_cast<size_t>(3 * G) * sizeof(int32_t));

    for (GroupMember* m : order) m->fresh = false;
    members_ = order;
    I.R = R;
    I.NNZ = NNZ;
    I.tiles = R / kTile;
    I.chunks = chunks;
    I.G = G;
    I.max_row_nnz = maxnz;
    I.dirty = false;
    I.eager_cycles = 0;
    ++repacks;
  }
  if (members_.empty()) return;

  // Filter scalings of this cycle.
  double* cd_h = I.cd_h.as<double>();
  for (int p = 0; p < I.G; ++p) {
    const GroupMember* m = members_[p];
    filter_scaling(m->cutoff, m->g.upper, &cd_h[2 * p], &cd_h[2 * p + 1]);
  }

  auto body = [&] {
    const int G = I.G;
    const int64_t R = I.R;
    const size_t bb = static_cast<size_t>(b) * b;
    double* B[kBlocks];
    for (int i = 0; i < kBlocks; ++i) B[i] = I.blk[i].as<double>();
    int32_t* info = I.info.as<int32_t>();
    FE_CHECK_CUDA(cudaMemcpyAsync(I.cd.get(), I.cd_h.as<double>(), 2 * G * sizeof(double),
                                  cudaMemcpyHostToDevice, s));
    // 2. filter: step k's result in ring slot k mod 3 (FP32 groups: an FP32 ring,
    // the result widened into slot 1 of the FP64 blocks)
    int res = static_cast<int>(degree_ % 3);
    if (fp32_) {
      group_rescale_f32(I.rowptr.as<int32_t>(), I.colind.as<int32_t>(), I.plain.as<double>(),
                        I.scaled32.as<float>(), R, I.tile_member.as<int32_t>(),
                        I.cd.as<double>(), s);
      float* F[3] = {I.f32[0].as<float>(), I.f32[1].as<float>(), I.f32[2].as<float>()};
      convert<double, float>(B[0], b, F[0], b, R, b, s);
      csr_spmm<float>(I.op_scaled, F[0], b, F[1], b, nullptr, 0, b, 1.0, 0.0, 0.0, s);
      for (int64_t k = 2; k <= degree_; ++k) {
        const int prev = static_cast<int>((k - 2) % 3), cur = static_cast<int>((k - 1) % 3),
                  next = static_cast<int>(k % 3);
        csr_spmm<float>(I.op_scaled, F[cur], b, F[next], b, F[prev], b, b, 2.0, 0.0, -1.0, s);
      }
      convert<float, double>(F[res], b, B[1], b, R, b, s);
      res = 1;
    } else {
      group_rescale(I.rowptr.as<int32_t>(), I.colind.as<int32_t>(), I.plain.as<double>(),
                    I.scaled.as<double>(), R, I.tile_member.as<int32_t>(), I.cd.as<double>(),
                    s);
      csr_spmm<double>(I.op_scaled, B[0], b, B[1], b, nullptr, 0, b, 1.0, 0.0, 0.0, s);
      for (int64_t k = 2; k <= degree_; ++k) {
        const int prev = static_cast<int>((k - 2) % 3), cur = static_cast<int>((k - 1) % 3),
                  next = static_cast<int>(k % 3);
        csr_spmm<double>(I.op_scaled, B[cur], b, B[next], b, B[prev], b, b, 2.0, 0.0, -1.0, s);
      }
    }
    // 3. Cholesky QR twice, ending in a slot other than 0 (slot 0 receives X)
    const int s1 = res == 0 ? 1 : (res == 1 ? 2 : 1);
    const int s2 = res == 0 ? 2 : res;
    auto cholqr = [&](int src, int dst, int32_t* inf) {
      gram_partial_dmma_ranges(B[src], b, B[src], b, static_cast<int>(b), static_cast<int>(b),
                               static_cast<int>(I.chunks), I.chunk_rows.as<int64_t>(), true,
                               I.gpart.as<double>(), s);
      group_gram_reduce(I.gpart.as<double>(), static_cast<int>(b), static_cast<int>(b), G,
                        I.member_chunks.as<int32_t>(), true, I.Gm.as<double>(), bb, s);
      if (chol_inv_small_fits(b)) {
        chol_inv_upper_batched(I.Gm.as<double>(), b, b, bb, I.Rinv.as<double>(), b, bb, G, inf,
                               s);
      } else {
        potrf_upper_batched(I.Gm.as<double>(), b, b, bb, G, inf, s);
        trinv_upper_batched(I.Gm.as<double>(), b, I.Rinv.as<double>(), b, b, bb, G, s);
      }
      rotate_dmma(B[src], b, I.Rinv.as<double>(), b, B[dst], b, R, b, b, 1.0, 0.0, s, true,
                  I.tile_member.as<int32_t>(), bb);
    };
    cholqr(res, s1, info);
    cholqr(s1, s2, info + G);
    const int basis = s2;
    // 4. Rayleigh-Ritz
    csr_spmm<double>(I.op_plain, B[basis], b, B[3], b, nullptr, 0, b, 1.0, 0.0, 0.0, s);
    gram_partial_dmma_ranges(B[basis], b, B[3], b, static_cast<int>(b), static_cast<int>(b),
                             static_cast<int>(I.chunks), I.chunk_rows.as<int64_t>(), false,
                             I.gpart.as<double>(), s);
    group_gram_reduce(I.gpart.as<double>(), static_cast<int>(b), static_cast<int>(b), G,
                      I.member_chunks.as<int32_t>(), false, I.Gm.as<double>(), bb, s);
    symmetrize_batched(I.Gm.as<double>(), b, b, bb, G, s);
    syevd_batched_uniform(G, b, I.Gm.as<double>(), b, I.theta.as<double>(), I.Q.as<double>(),
                          info + 2 * G, I.syevd_ws.get(), I.syevd_ws.bytes(), s);
    rotate_dmma(B[basis], b, I.Q.as<double>(), b, B[0], b, R, b, b, 1.0, 0.0, s, false,
                I.tile_member.as<int32_t>(), bb);
    rotate_dmma(B[3], b, I.Q.as<double>(), b, B[4], b, R, b, b, 1.0, 0.0, s, false,
                I.tile_member.as<int32_t>(), bb);
    group_residuals(B[4], B[0], b, static_cast<int>(b), static_cast<int>(I.chunks),
                    I.chunk_rows.as<int64_t>(), I.chunk_member.as<int32_t>(), G,
                    I.member_chunks.as<int32_t>(), I.theta.as<double>(), I.rpart.as<double>(),
                    I.rel.as<double>(), s);
    // 5. results of the cycle to the host
    FE_CHECK_CUDA(cudaMemcpyAsync(I.theta_h.as<double>(), I.theta.get(), G * b * sizeof(double),
                                  cudaMemcpyDeviceToHost, s));
    FE_CHECK_CUDA(cudaMemcpyAsync(I.rel_h.as<double>(), I.rel.get(), G * b * sizeof(double),
                                  cudaMemcpyDeviceToHost, s));
    FE_CHECK_CUDA(cudaMemcpyAsync(I.info_h.as<int32_t>(), I.info.get(), 3 * G * sizeof(int32_t),
                                  cudaMemcpyDeviceToHost, s));
  };

  // The first cycle after a repack runs eagerly (it also sets kernel attributes and
  // caches launch choices); the second is captured into a graph that later cycles
  // replay.
  if (I.eager_cycles < 1) {
    body();
    ++I.eager_cycles;
  } else {
    if (!I.exec) {
      FE_CHECK_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      try {
        body();
      } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(s, &g);
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        throw;
      }
      FE_CHECK_CUDA(cudaStreamEndCapture(s, &I.graph));
      FE_CHECK_CUDA(cudaGraphInstantiate(&I.exec, I.graph, 0));
    }
    FE_CHECK_CUDA(cudaGraphLaunch(I.exec, s));
    ++graph_replays;
  }
  launched_ = true;
}

void ChebGroup::finish_cycle(std::vector<GroupMember*>& done) {
  if (!launched_) return;
  launched_ = false;
  FE_CHECK_CUDA(cudaStreamSynchronize(stream_));
  AllocOn on(stream_);
  ++cycles;
  bool carried = false;
  Impl& I = *impl_;
  const int64_t b = width_;
  const double* theta = I.theta_h.as<double>();
  const double* rel = I.rel_h.as<double>();
  const int32_t* info = I.info_h.as<int32_t>();
  std::vector<GroupMember*> keep;
  for (int p = 0; p < I.G; ++p) {
    GroupMember* m = members_[p];
    ++m->iterations;
    if (fp32_) ++m->fp32_iterations;
    const double* th = theta + static_cast<int64_t>(p) * b;
    const double* rl = rel + static_cast<int64_t>(p) * b;
    bool finite = true;
    for (int64_t j = 0; j < b; ++j) finite = finite && std::isfinite(th[j]) && std::isfinite(rl[j]);
    std::string fail;
    int rc = FE_OK;
    if (info[p] != 0 || info[I.G + p] != 0) {
      rc = FE_ERR_NOT_SPD;
      fail = "ChebyshevSolver: Cholesky QR failed during filtering.";
    } else if (info[2 * I.G + p] != 0 || !finite) {
      rc = FE_ERR_NONFINITE;
      fail = "ChebyshevSolver: non-finite Ritz values or residuals.";
    }
    double worst = 0.0;
    for (int64_t j = 0; j < m->g.nev; ++j) worst = std::max(worst, rl[j]);
    const bool converged = rc == FE_OK && worst <= m->g.tol;
    if (fp32_ && rc == FE_OK && !converged && m->iterations < m->g.maxiter) {
      // Leave the FP32 filter at its residual floor, or when it stops reducing the
      // worst residual (no 30 % gain over three cycles), as the mixed single solve.
      m->worst_history.push_back(worst);
      const size_t h = m->worst_history.size();
      const bool stalled = h >= 4 && worst > 0.7 * m->worst_history[h - 4];
      if (worst <= std::max(m->g.tol, m->g.mixed_switch) || stalled) {
        if (m->g.ritz_bounds) m->cutoff = std::min(th[b - 1], m->g.ritz_cutoff_cap);
        m->carry.resize(static_cast<size_t>(m->n_pad) * b * sizeof(double));
        FE_CHECK_CUDA(cudaMemcpyAsync(m->carry.get(), I.blk[0].as<double>() + m->row0 * b,
                                      static_cast<size_t>(m->n_pad) * b * sizeof(double),
                                      cudaMemcpyDeviceToDevice, stream_));
        m->switched = true;
        carried = true;
        done.push_back(m);
        continue;
      }
    }
    if (rc == FE_OK && !converged && m->iterations < m->g.maxiter) {
      // bounds=ritz: damp up to the largest Ritz value of the subspace, capped so the
      // amplification at `lower` stays within the requested one.
      if (m->g.ritz_bounds) m->cutoff = std::min(th[b - 1], m->g.ritz_cutoff_cap);
      keep.push_back(m);
      continue;
    }
    m->rc = rc;
    m->error = fail;
    m->converged = converged;
    m->eigenvalues.resize(m->g.nev);
    m->residuals.resize(m->g.nev);
    for (int64_t j = 0; j < m->g.nev; ++j) {
      m->eigenvalues[j] = m->g.sign * th[j];
      m->residuals[j] = rl[j];
    }
    if (rc == FE_OK && m->want_vectors) {
      // Ritz block rows of the member (row-major, width b) -> column-major n x nev.
      const int64_t n = m->A->rows;
      std::vector<double> rows(static_cast<size_t>(n) * b);
      FE_CHECK_CUDA(cudaMemcpy(rows.data(), I.blk[0].as<double>() + m->row0 * b,
                               rows.size() * sizeof(double), cudaMemcpyDeviceToHost));
      m->vectors.resize(static_cast<size_t>(n) * m->g.nev);
      for (int64_t j = 0; j < m->g.nev; ++j)
        for (int64_t i = 0; i < n; ++i)
          m->vectors[static_cast<size_t>(j) * n + i] = rows[static_cast<size_t>(i) * b + j];
    }
    m->seconds =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - m->t_join).count();
    done.push_back(m);
  }
  if (carried) FE_CHECK_CUDA(cudaStreamSynchronize(stream_));
  if (keep.size() != members_.size()) {
    members_ = keep;
    I.dirty = true;
  }
  if (!joining_.empty()) I.dirty = true;
}

}  // namespace fe

// ---------------------------------------------------------------------------
// C ABI: a batch of standard Chebyshev problems solved together in groups (one
// group per width and degree, the groups' cycles overlapping on their streams).
// ---------------------------------------------------------------------------
extern "C" int fe_grouped_chebyshev(int32_t count, const fe_csr_t* A, const char* const* options,
                                    double* const* eigenvalues, double* const* residual_norms,
                                    double* const* eigenvectors, double* stats) {
  return fe::guarded("fe_grouped_chebyshev", [&] {
    FE_REQUIRE(count > 0 && A && options && eigenvalues && residual_norms,
               "null or empty batch");
    const int device = A[0] ? A[0]->m.device : 0;
    FE_CHECK_CUDA(cudaSetDevice(device));
    // groups before members: a member's carried block is freed on its group's stream
    std::vector<std::unique_ptr<fe::ChebGroup>> groups;
    std::vector<fe::GroupMember> members(count);
    for (int32_t p = 0; p < count; ++p) {
      FE_REQUIRE(A[p] && A[p]->m.device == device, "null CSR handle or operator on another device");
      FE_REQUIRE(eigenvalues[p] && residual_norms[p], "null result arrays");
      fe::GroupMember& m = members[p];
      m.A = &A[p]->m;
      m.want_vectors = eigenvectors && eigenvectors[p];
      fe::chebyshev_group_setup(*m.A, options[p], m.g);
    }
    // one group per (width, degree, filter precision); mixed members start in the
    // FP32-filter group and move to the FP64 one at their floor
    auto group_for = [&](const fe::GroupMember& m, bool fp32) {
      for (auto& x : groups)
        if (x->width() == m.g.width && x->degree() == m.g.degree && x->fp32_filter() == fp32)
          return x.get();
      groups.emplace_back(new fe::ChebGroup(device, m.g.width, m.g.degree, fp32));
      return groups.back().get();
    };
    for (auto& m : members) group_for(m, m.g.mixed)->join(&m);
    std::vector<fe::GroupMember*> done, moving;
    int64_t cycles = 0, replays = 0, repacks = 0;
    while (true) {
      bool any = false;
      for (auto& g : groups) {
        if (g->empty()) continue;
        g->launch_cycle();
        any = true;
      }
      if (!any) break;
      moving.clear();
      for (size_t i = 0; i < groups.size(); ++i) {
        done.clear();
        groups[i]->finish_cycle(done);
        for (fe::GroupMember* m : done)
          if (m->switched) moving.push_back(m);
      }
      for (fe::GroupMember* m : moving) group_for(*m, false)->join(m);
    }
    for (auto& g : groups) {
      cycles += g->cycles;
      replays += g->graph_replays;
      repacks += g->repacks;
    }
    const auto first_error = [&]() -> const fe::GroupMember* {
      for (const auto& m : members)
        if (m.rc != FE_OK) return &m;
      return nullptr;
    }();
    for (int32_t p = 0; p < count; ++p) {
      const fe::GroupMember& m = members[p];
      std::copy(m.eigenvalues.begin(), m.eigenvalues.end(), eigenvalues[p]);
      std::copy(m.residuals.begin(), m.residuals.end(), residual_norms[p]);
      if (m.want_vectors && !m.vectors.empty())
        std::copy(m.vectors.begin(), m.vectors.end(), eigenvectors[p]);
      if (stats) {
        double* st = stats + static_cast<int64_t>(p) * FE_GROUP_STATS;
        st[0] = static_cast<double>(m.iterations);
        st[1] = m.converged ? 0.0 : 1.0;
        st[2] = m.seconds;
        st[3] = static_cast<double>(m.g.width);
        st[4] = m.g.lower;
        st[5] = m.g.upper;
        st[6] = static_cast<double>(cycles);
        st[7] = static_cast<double>(replays);
        st[8] = static_cast<double>(repacks);
        st[9] = static_cast<double>(m.rc);
        st[10] = static_cast<double>(m.fp32_iterations);
      }
    }
    if (first_error)
      throw fe::Error(first_error->rc, "problem " +
                                           std::to_string(first_error - members.data()) + ": " +
                                           first_error->error);
  });
}
