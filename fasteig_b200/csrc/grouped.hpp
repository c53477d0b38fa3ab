// Grouped Chebyshev engine (extension): many standard eigenproblems advance
// together, one filter cycle at a time, in grouped kernels over one concatenated
// block-diagonal operator. Requests join and leave between cycles (continuous
// batching); while the membership stays the same each cycle replays one CUDA
// graph.
//
// Each member runs the reference's ChebyshevSolver cycle (src/ChebyshevSolver.cpp:
// 145-205: filter, Cholesky QR, Rayleigh-Ritz, residual check), with the whole
// subspace filtered every cycle (this backend's soft locking) and the member's
// width rounded up to a multiple of 32 columns. A group filters in FP64 or, for
// precision=mixed members until their FP32 floor, in FP32 (everything after the
// filter stays FP64); a mixed member at its floor moves to the FP64 group of its
// width with its Ritz block.
#pragma once

#include "device.hpp"

#include <chrono>
#include <memory>
#include <string>
#include <vector>

namespace fe {

struct GroupSetup {
  int64_t n = 0, nev = 0, width = 0, degree = 0, maxiter = 0;
  double tol = 0, sign = 1, lower = 0, upper = 0, amplification = 1e3;
  // filter cutoffs: the reference's fixed one (amplification 1e3 at `lower`) and,
  // for bounds=ritz, the cap at the requested amplification
  double reference_cutoff = 0, ritz_cutoff_cap = 0;
  bool ritz_bounds = false, host_init = true;
  bool mixed = false;          // FP32 filter until the FP32 floor, then FP64
  double mixed_switch = 4e-6;  // the floor: leave FP32 when the worst residual is below
  unsigned seed = 1;
};

// Whether a request may run in a group (standard Chebyshev, FP64 or mixed, soft
// locking, width <= 512), with its group key (width, degree). With require_flag the
// option string must also ask for it (group=1).
bool chebyshev_group_key(const Csr& A, const Csr* B, const char* options, bool require_flag,
                         int64_t* width, int64_t* degree, bool* mixed = nullptr);
// Option checks and the Lanczos spectral bounds of one member (its own stream).
void chebyshev_group_setup(const Csr& A, const char* options, GroupSetup& g);
// Device memory one member adds to its group (blocks, operator copy, workspaces),
// including the transient of a repack; `mixed` adds the FP32 filter blocks and the
// Ritz block carried to the FP64 group.
size_t group_member_bytes(const Csr& A, int64_t width, bool mixed = false);

struct GroupMember {
  const Csr* A = nullptr;
  GroupSetup g;
  void* tag = nullptr;
  bool want_vectors = false;
  // results, valid once the member left its group
  std::vector<double> eigenvalues, residuals, vectors;  // vectors: column-major n x nev
  int64_t iterations = 0, fp32_iterations = 0;
  bool converged = false;
  // set when a mixed member leaves its FP32 group at the floor: it is not done and
  // joins the FP64 group of its width with `carry` (its n_pad x width FP64 Ritz rows)
  bool switched = false;
  DeviceBuffer carry;
  std::vector<double> worst_history;
  int rc = FE_OK;
  std::string error;
  double seconds = 0;
  // engine state
  int64_t row0 = 0, n_pad = 0, nz0 = 0, chunk0 = 0, chunks = 0;
  bool fresh = true;
  double cutoff = 0;
  std::chrono::steady_clock::time_point t_join;
};

class ChebGroup {
 public:
  ChebGroup(int device, int64_t width, int64_t degree, bool fp32_filter = false);
  ~ChebGroup();
  ChebGroup(const ChebGroup&) = delete;
  ChebGroup& operator=(const ChebGroup&) = delete;

  int64_t width() const { return width_; }
  int64_t degree() const { return degree_; }
  bool fp32_filter() const { return fp32_; }
  bool empty() const { return members_.empty() && joining_.empty(); }
  size_t size() const { return members_.size() + joining_.size(); }
  cudaStream_t stream() const { return stream_; }

  // The member enters at the next cycle (its setup already done).
  void join(GroupMember* m);
  // Queue one filter cycle of every member on the group's stream (repacking first
  // when members joined or left) ...
  void launch_cycle();
  // ... then wait for it and move the members that finished (converged, at
  // maxiter, or failed) to `done`; in an FP32-filter group, members at their FP32
  // floor leave to `done` too with `switched` set (not finished).
  void finish_cycle(std::vector<GroupMember*>& done);
  // Device failure of a whole cycle: every member leaves with this error.
  void fail_all(int rc, const std::string& error, std::vector<GroupMember*>& done);

  int64_t cycles = 0, graph_replays = 0, repacks = 0;

 private:
  struct Impl;
  std::unique_ptr<Impl> impl_;
  int device_;
  int64_t width_, degree_;
  bool fp32_;
  cudaStream_t stream_ = nullptr;
  std::vector<GroupMember*> members_, joining_;
  bool launched_ = false;
};

// Grouped kernels (group_kernels.cu).
// Concatenated block-diagonal operator: rows of a member at row0 (padded to n_pad
// empty rows), its entries at nz0, columns shifted by row0, values times `sign`.
void group_pack_member(const Csr& A, int64_t row0, int64_t n_pad, int64_t nz0, double sign,
                       int32_t* cat_rowptr, int32_t* cat_colind, double* cat_plain,
                       cudaStream_t s);
// Rows of A whose stored diagonal count is not exactly one (device count).
void csr_count_bad_diagonals(const Csr& A, int32_t* count, cudaStream_t s);
// scaled = c_p * plain + d_p * I on the rows of member p (tile_member: row tile ->
// member, cd: [c_0, d_0, c_1, d_1, ...]).
void group_rescale(const int32_t* rowptr, const int32_t* colind, const double* plain,
                   double* scaled, int64_t rows, const int32_t* tile_member, const double* cd,
                   cudaStream_t s);
void group_rescale_f32(const int32_t* rowptr, const int32_t* colind, const double* plain,
                       float* scaled, int64_t rows, const int32_t* tile_member, const double* cd,
                       cudaStream_t s);
// Sum of the Gram partials of each member's chunks into its k x m matrix
// (column-major, ld k, `stride` doubles apart).
void group_gram_reduce(const double* partial, int k, int m, int members,
                       const int32_t* member_chunks, bool symmetric, double* G, int64_t stride,
                       cudaStream_t s);
// Relative residuals ||AX_j - theta_j X_j|| / ((1 + |theta_j|) ||X_j||) of every
// member's columns (theta, rel: members x width).
void group_residuals(const double* AX, const double* X, int64_t ld, int width, int chunks,
                     const int64_t* chunk_rows, const int32_t* chunk_member, int members,
                     const int32_t* member_chunks, const double* theta, double* partial,
                     double* rel, cudaStream_t s);

}  // namespace fe
