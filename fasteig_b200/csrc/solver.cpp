// Device-resident solver drivers of the B200 backend.
//
// The reference runs each solver against its executor abstraction
// (include/core/Executor.hpp:22-47) with host-synchronous orchestration: every
// transpose_multiply, column_norms, potrf info and projected eigensolve returns
// to the host (src/gpu/CudaMultiVector.cpp:389-405,455-473;
// src/core/Orthogonalization.cpp:211-243). Here all n-by-block state stays in
// HBM; per iteration only the k Ritz values, k relative residuals and the
// Cholesky status word come back to the host, which is what the locking and
// convergence logic of the reference needs.
//
// Chebyshev follows ChebyshevSolver::solve (src/ChebyshevSolver.cpp:67-221).
// Precision: "fp64" runs every block in FP64 (the plain path); "mixed" runs the
// filter, SpMMs and rotations on FP32 blocks with FP64-accumulated Grams, FP64
// Cholesky and an FP64 projected eigensolve, then switches the block to FP64 for
// the final sweeps once the FP32 residual floor is reached; those sweeps filter
// through an FP32 correction recurrence that keeps FP64 accuracy (refined_filter).


#include <chrono>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <random>
#include <sstream>
#include <type_traits>

#include "device.hpp"
#include "grouped.hpp"
#include "tridiag.hpp"

namespace fe {
namespace {

std::string lower(std::string s) {
  for (auto& c : s) c = static_cast<char>(std::tolower(static_cast<unsigned char>(c)));
  return s;
}

// Options with the reference's keys and defaults (include/fasteig_options.hpp:102-118),
// plus this backend's extensions.
struct Options {
  std::string solver = "chebyshev";
  std::string which = "sr";
  int64_t nev = 10;
  int64_t maxiter = 1000;
  int64_t maxdim = 0;
  int64_t maxblks = 10;
  int64_t degree = 10;
  int64_t blksize = 1;
  double tol = 1.0e-8;
  bool has_seed = false;
  unsigned seed = 1;
  int verbosity = 0;
  int64_t print_every = 0;  // LanczosSolver: convergence checked every print_every steps (0: 5)
  // extensions
  std::string precision = "fp64";  // fp64 | mixed
  int64_t block = 0;               // Chebyshev subspace capacity override (0 = reference rule)
  std::string bounds = "reference";  // reference | ritz
  double amplification = 1.0e3;    // filter amplification cap at the lower bound
  std::string init = "host";       // host (std::mt19937, bit-exact) | device
  double mixed_switch = 4.0e-6;    // FP32 -> FP64 switch when max residual <= this
  bool tensor_cores = true;        // FP32 Grams/rotations on tcgen05 (3xTF32)
  std::string precond = "none";    // none | jacobi (LOBPCG / Davidson corrections W = T R)
  std::string locking = "soft";    // Chebyshev: soft (reference) | hard
  int64_t tail_degree = 0;         // Chebyshev mixed: filter degree of the FP64 cycles (0 = degree)
  int64_t tail_guard = 0;          // Chebyshev mixed: columns past nev in the FP64 cycles (0 = all)
  std::string tail_rr = "split";   // Chebyshev mixed FP64 cycles: Y^T A Y as split | fp64
  int64_t inject_wait_timeout = 0;  // test hook: status code of a forced bounded-wait timeout
  bool group = false;  // request server: Chebyshev request may run in a grouped lane
  // Chebyshev hard locking: Rayleigh-Ritz with the Cholesky QR rotation folded in
  // ("fused", the default of precision=mixed) or Cholesky QR then Rayleigh-Ritz as
  // the reference orders them ("cholqr", the default of precision=fp64).
  std::string rr = "";
  // Chebyshev mixed: filter of the FP64 cycles, "refined" (FP32 correction recurrence,
  // FP64 accuracy) or "fp64" (FP64 SpMMs).
  std::string tail_filter = "refined";

  void parse(const char* text) {
    if (!text) return;
    std::string s(text);
    for (auto& c : s)
      if (c == ';' || c == ',') c = '\n';
    std::istringstream in(s);
    std::string line;
    while (std::getline(in, line)) {
      auto eq = line.find('=');
      if (eq == std::string::npos) {
        // also accept "key value" deck lines
        std::istringstream ls(line);
        std::string k, v;
        if (!(ls >> k)) continue;
        if (!(ls >> v)) throw Error(FE_ERR_INVALID, "option without value: " + k);
        set(lower(k), v);
        continue;
      }
      auto trim = [](std::string x) {
        const auto b = x.find_first_not_of(" \t\r");
        const auto e = x.find_last_not_of(" \t\r");
        return b == std::string::npos ? std::string() : x.substr(b, e - b + 1);
      };
      const std::string k = lower(trim(line.substr(0, eq)));
      const std::string v = trim(line.substr(eq + 1));
      if (k.empty()) continue;
      set(k, v);
    }
  }

  void set(const std::string& k, const std::string& v) {
    auto as_int = [&](const std::string& x) {
      size_t pos = 0;
      const long long r = std::stoll(x, &pos);
      if (pos != x.size()) throw Error(FE_ERR_INVALID, "invalid integer for " + k + ": " + x);
      return static_cast<int64_t>(r);
    };
    auto as_double = [&](const std::string& x) {
      size_t pos = 0;
      const double r = std::stod(x, &pos);
      if (pos != x.size()) throw Error(FE_ERR_INVALID, "invalid number for " + k + ": " + x);
      return r;
    };
    if (k == "solver") solver = lower(v);
    else if (k == "which") which = lower(v);
    else if (k == "nev") nev = as_int(v);
    else if (k == "maxiter") maxiter = as_int(v);
    else if (k == "maxdim") maxdim = as_int(v);
    else if (k == "maxblks") maxblks = as_int(v);
    else if (k == "degree") degree = as_int(v);
    else if (k == "blksize") blksize = as_int(v);
    else if (k == "tol") tol = as_double(v);
    else if (k == "seed") {
      const long long sd = std::stoll(v);
      if (sd < 0) has_seed = false;
      else if (sd > static_cast<long long>(std::numeric_limits<unsigned>::max()))
        throw Error(FE_ERR_INVALID, "seed out of range for unsigned int");
      else { has_seed = true; seed = static_cast<unsigned>(sd); }
    } else if (k == "verbosity") verbosity = static_cast<int>(as_int(v));
    else if (k == "precision") precision = lower(v);
    else if (k == "block") block = as_int(v);
    else if (k == "bounds") bounds = lower(v);
    else if (k == "amplification") amplification = as_double(v);
    else if (k == "init") init = lower(v);
    else if (k == "mixed_switch") mixed_switch = as_double(v);
    else if (k == "tensor_cores") tensor_cores = as_int(v) != 0;
    else if (k == "group") group = as_int(v) != 0;
    else if (k == "tail_degree") tail_degree = as_int(v);
    else if (k == "tail_rr") {
      tail_rr = lower(v);
      if (tail_rr != "split" && tail_rr != "fp64")
        throw Error(FE_ERR_INVALID, "tail_rr must be split or fp64");
    } else if (k == "tail_guard") {
      tail_guard = as_int(v);
      if (tail_guard < 0) throw Error(FE_ERR_INVALID, "tail_guard must be >= 0");
    }
    else if (k == "inject_wait_timeout") inject_wait_timeout = as_int(v);
    else if (k == "tail_filter") {
      tail_filter = lower(v);
      if (tail_filter != "refined" && tail_filter != "fp64")
        throw Error(FE_ERR_INVALID, "tail_filter must be refined or fp64");
    } else if (k == "rr") {
      rr = lower(v);
      if (rr != "fused" && rr != "cholqr") throw Error(FE_ERR_INVALID, "rr must be fused or cholqr");
    }
    else if (k == "locking") {
      locking = lower(v);
      if (locking != "soft" && locking != "hard")
        throw Error(FE_ERR_INVALID, "locking must be soft or hard");
    } else if (k == "precond") {
      precond = lower(v);
      if (precond != "none" && precond != "jacobi")
        throw Error(FE_ERR_INVALID, "precond must be none or jacobi");
    }
    else if (k == "print_every") print_every = as_int(v);
    else if (k == "logfile" || k == "output_format" || k == "gpu_backend" || k == "shift" ||
             k == "n") {
      // accepted for deck compatibility; no effect on this backend
    } else {
      throw Error(FE_ERR_INVALID, "unknown option: " + k);
    }
  }
  unsigned seed_or_default() const { return has_seed ? seed : 1u; }
};

struct Stats {
  double iterations = 0, status = 0, seconds = 0, fp32_iterations = 0, fp64_iterations = 0;
  double spmm_launches = 0, lower = 0, upper = 0;
  // device time per phase (ms, CUDA events on the solver stream)
  double filter_ms = 0, ortho_ms = 0, rr_ms = 0, precise_grams = 0;
};

// Events bracketing the phases of one filter cycle.
struct PhaseEvents {
  cudaEvent_t e[4] = {nullptr, nullptr, nullptr, nullptr};
  PhaseEvents() {
    for (auto& x : e) FE_CHECK_CUDA(cudaEventCreate(&x));
  }
  ~PhaseEvents() {
    for (auto& x : e)
      if (x) cudaEventDestroy(x);
  }
  void record(int i, cudaStream_t s) { FE_CHECK_CUDA(cudaEventRecord(e[i], s)); }
  // after a stream sync
  void accumulate(Stats& st) {
    float a = 0, b = 0, c = 0;
    FE_CHECK_CUDA(cudaEventElapsedTime(&a, e[0], e[1]));
    FE_CHECK_CUDA(cudaEventElapsedTime(&b, e[1], e[2]));
    FE_CHECK_CUDA(cudaEventElapsedTime(&c, e[2], e[3]));
    st.filter_ms += a;
    st.ortho_ms += b;
    st.rr_ms += c;
  }
};

// One solve's stream. While it lives, this thread's DeviceBuffers are allocated
// from the device's stream-ordered pool on its stream (buffers declared after the
// Context are released before it). Streams are kept for reuse (per device, shared by
// all threads).
struct ContextResources {
  int device;
  cudaStream_t stream;
};
std::mutex g_ctx_mutex;
std::vector<ContextResources> g_ctx_free;

class Context {
 public:
  cudaStream_t stream = nullptr;
  Context() {
    FE_CHECK_CUDA(cudaGetDevice(&device_));
    retain_pool_memory(device_);
    {
      std::lock_guard<std::mutex> lock(g_ctx_mutex);
      for (size_t i = 0; i < g_ctx_free.size(); ++i) {
        if (g_ctx_free[i].device == device_) {
          stream = g_ctx_free[i].stream;
          g_ctx_free.erase(g_ctx_free.begin() + static_cast<std::ptrdiff_t>(i));
          break;
        }
      }
    }
    if (!stream) FE_CHECK_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    prev_alloc_ = alloc_stream();
    alloc_stream() = stream;
  }
  ~Context() {
    alloc_stream() = prev_alloc_;
    if (!stream) return;
    if (cudaStreamSynchronize(stream) == cudaSuccess) {
      std::lock_guard<std::mutex> lock(g_ctx_mutex);
      g_ctx_free.push_back({device_, stream});
    } else {
      cudaStreamDestroy(stream);
    }
  }
  Context(const Context&) = delete;
  Context& operator=(const Context&) = delete;
  void sync() { FE_CHECK_CUDA(cudaStreamSynchronize(stream)); }
  template <typename T>
  void to_host(T* dst, const T* src, size_t count) {
    FE_CHECK_CUDA(cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyDeviceToHost, stream));
  }
  template <typename T>
  void to_device(T* dst, const T* src, size_t count) {
    FE_CHECK_CUDA(cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyHostToDevice, stream));
  }

 private:
  cudaStream_t prev_alloc_ = nullptr;
  int device_ = 0;
};

// Host std::mt19937 draws in the reference's column-major order
// (Executor::create_random_multivector, src/core/Executor.cpp:44-62), scattered into
// a row-major host staging array and uploaded.
template <typename T>
void random_block_host(Context& ctx, Block<T>& X, int64_t cols, unsigned seed) {
  std::mt19937 rng(seed);
  std::uniform_real_distribution<double> dist(-1.0, 1.0);
  std::vector<T> host(static_cast<size_t>(X.n) * X.ld, T(0));
  for (int64_t j = 0; j < cols; ++j)
    for (int64_t i = 0; i < X.n; ++i) host[static_cast<size_t>(i) * X.ld + j] = static_cast<T>(dist(rng));
  FE_CHECK_CUDA(cudaMemcpyAsync(X.data(), host.data(), host.size() * sizeof(T),
                                cudaMemcpyHostToDevice, ctx.stream));
  ctx.sync();
}

// -------------------------------------------------------------------------
// Lanczos spectral bounds: estimate_bounds_with_executor (src/ChebyshevSolver.cpp:26-49)
// built on KrylovSubspace::build_one (src/core/KrylovSubspace.cpp:125-259) with
// two-pass classical reorthogonalization; FP64 on the device, the steps x steps
// tridiagonal eigensolve on the host (as CudaLanczosWorkspace returns its snapshot).
// -------------------------------------------------------------------------
void lanczos_bounds(Context& ctx, const Csr& A, double sign, unsigned seed, bool host_init,
                    double& lower_out, double& upper_out) {
  const int64_t n = A.rows;
  const int64_t steps = std::min<int64_t>(20, n);
  cudaStream_t s = ctx.stream;
  DeviceBuffer Vb(static_cast<size_t>(n) * steps * sizeof(double));  // row-major n x steps
  DeviceBuffer f(n * sizeof(double)), w(n * sizeof(double));
  DeviceBuffer h(steps * sizeof(double)), hs(steps * sizeof(double)), nrm(sizeof(double));
  const size_t gws = std::max(gram_workspace_bytes(n, steps, 1), residual_workspace_bytes(n, 1));
  DeviceBuffer ws(std::max<size_t>(gws, 64));
  double* V = Vb.as<double>();
  const int64_t ld = steps;
  if (host_init) {
    std::mt19937 rng(seed);
    std::uniform_real_distribution<double> dist(-1.0, 1.0);
    std::vector<double> v(n);
    for (auto& x : v) x = dist(rng);
    ctx.to_device(f.as<double>(), v.data(), n);
  } else {
    fill_uniform<double>(f.as<double>(), 1, n, 1, seed, s);
  }
  std::vector<double> T(static_cast<size_t>(steps) * steps, 0.0);
  auto norm = [&](const double* x) {
    residual_norms<double>(nullptr, x, nullptr, 1, n, 1, nullptr, nullptr, 0, nullptr,
                           nrm.as<double>(), nullptr, ws.get(), ws.bytes(), s, 0);
    double r = 0;
    ctx.to_host(&r, nrm.as<double>(), 1);
    ctx.sync();
    return r;
  };
  // Two-pass classical Gram-Schmidt of src against V[:, :k] into f; returns h[k-1].
  auto orthogonalize = [&](int64_t k, const double* src) {
    vec_axpby(n, 1.0, src, 1, 0.0, f.as<double>(), 1, s);
    if (k == 0) return 0.0;
    gram<double>(V, ld, f.as<double>(), 1, n, k, 1, h.as<double>(), k, ws.get(), ws.bytes(), s);
    rotate<double>(V, ld, h.as<double>(), k, f.as<double>(), 1, n, k, 1, -1.0, 1.0, s);
    gram<double>(V, ld, f.as<double>(), 1, n, k, 1, hs.as<double>(), k, ws.get(), ws.bytes(), s);
    rotate<double>(V, ld, hs.as<double>(), k, f.as<double>(), 1, n, k, 1, -1.0, 1.0, s);
    double a = 0, b = 0;
    ctx.to_host(&a, h.as<double>() + k - 1, 1);
    ctx.to_host(&b, hs.as<double>() + k - 1, 1);
    ctx.sync();
    return a + b;
  };
  double beta_next = 0.0;
  bool fast_done = false;
  // Fast path: the whole recurrence is queued with its scalars (norms, alpha)
  // kept on the device and read once at the end, instead of three host round
  // trips per step. A breakdown (a residual norm at rounding level, where the
  // reference restarts from a fresh random vector) is detected afterwards; the
  // recurrence is then redone step by step below from the same start vector.
  {
    DeviceBuffer f0(n * sizeof(double)), alphas(steps * sizeof(double)),
        betas((steps + 1) * sizeof(double));
    vec_axpby(n, 1.0, f.as<double>(), 1, 0.0, f0.as<double>(), 1, s);
    auto dnorm = [&](const double* x, double* out) {
      residual_norms<double>(nullptr, x, nullptr, 1, n, 1, nullptr, nullptr, 0, nullptr, out,
                             nullptr, ws.get(), ws.bytes(), s, 0);
    };
    for (int64_t it = 0; it < steps; ++it) {
      dnorm(f.as<double>(), betas.as<double>() + it);
      scale_by_inv(n, f.as<double>(), betas.as<double>() + it, V + it, ld, s);
      csr_spmm<double>(A, V + it, ld, w.as<double>(), 1, nullptr, 0, 1, sign, 0.0, 0.0, s);
      const int64_t k = it + 1;
      vec_axpby(n, 1.0, w.as<double>(), 1, 0.0, f.as<double>(), 1, s);
      gram<double>(V, ld, f.as<double>(), 1, n, k, 1, h.as<double>(), k, ws.get(), ws.bytes(), s);
      rotate<double>(V, ld, h.as<double>(), k, f.as<double>(), 1, n, k, 1, -1.0, 1.0, s);
      gram<double>(V, ld, f.as<double>(), 1, n, k, 1, hs.as<double>(), k, ws.get(), ws.bytes(),
                   s);
      rotate<double>(V, ld, hs.as<double>(), k, f.as<double>(), 1, n, k, 1, -1.0, 1.0, s);
      sum2(h.as<double>() + k - 1, hs.as<double>() + k - 1, alphas.as<double>() + it, s);
    }
    dnorm(f.as<double>(), betas.as<double>() + steps);
    std::vector<double> al(steps), be(steps + 1);
    ctx.to_host(al.data(), alphas.as<double>(), steps);
    ctx.to_host(be.data(), betas.as<double>(), steps + 1);
    ctx.sync();
    bool ok = true;
    for (int64_t it = 0; it < steps; ++it)
      ok = ok && std::isfinite(al[it]) && std::isfinite(be[it]) &&
           be[it] > std::numeric_limits<double>::epsilon();
    ok = ok && std::isfinite(be[steps]);
    if (ok) {
      for (int64_t it = 0; it < steps; ++it) {
        if (it != 0) {
          T[static_cast<size_t>(it - 1) * steps + it] = be[it];
          T[static_cast<size_t>(it) * steps + it - 1] = be[it];
        }
        T[static_cast<size_t>(it) * steps + it] = al[it];
      }
      beta_next = be[steps];
      fast_done = true;
    } else {
      vec_axpby(n, 1.0, f0.as<double>(), 1, 0.0, f.as<double>(), 1, s);
    }
  }
  if (!fast_done) {
    for (int64_t it = 0; it < steps; ++it) {
      bool restarted = false;
      double beta = norm(f.as<double>());
      if (!std::isfinite(beta)) throw Error(FE_ERR_NONFINITE, "Lanczos: non-finite residual norm");
      if (!(beta > std::numeric_limits<double>::epsilon())) {
        // restart_residual (src/core/KrylovSubspace.cpp:251-259)
        DeviceBuffer cand(n * sizeof(double));
        if (host_init) {
          std::mt19937 rng(seed + static_cast<unsigned>(it + 1));
          std::uniform_real_distribution<double> dist(-1.0, 1.0);
          std::vector<double> v(n);
          for (auto& x : v) x = dist(rng);
          ctx.to_device(cand.as<double>(), v.data(), n);
        } else {
          fill_uniform<double>(cand.as<double>(), 1, n, 1, seed + it + 1, s);
        }
        orthogonalize(it, cand.as<double>());
        restarted = true;
        beta = norm(f.as<double>());
        if (!(beta > std::numeric_limits<double>::epsilon()))
          throw Error(FE_ERR_NONFINITE, "Lanczos: breakdown, unable to generate new basis vector.");
      }
      vec_axpby(n, 1.0 / beta, f.as<double>(), 1, 0.0, V + it, ld, s);
      csr_spmm<double>(A, V + it, ld, w.as<double>(), 1, nullptr, 0, 1, sign, 0.0, 0.0, s);
      const double alpha = orthogonalize(it + 1, w.as<double>());
      beta_next = norm(f.as<double>());
      if (!std::isfinite(beta_next)) throw Error(FE_ERR_NONFINITE, "Lanczos: non-finite norm");
      const double rec_beta = restarted ? 0.0 : beta;
      if (it != 0) {
        T[static_cast<size_t>(it - 1) * steps + it] = rec_beta;
        T[static_cast<size_t>(it) * steps + it - 1] = rec_beta;
      }
      T[static_cast<size_t>(it) * steps + it] = alpha;
    }
  }
  std::vector<double> lam, Z;
  host_symmetric_eig(T, static_cast<int>(steps), lam, Z);
  double lo = std::numeric_limits<double>::infinity(), up = -lo;
  for (int64_t j = 0; j < steps; ++j) {
    // lanczos_absolute_residuals: rel*(1+|l|) = |beta_next * Z[m-1, j]|
    const double r = std::fabs(beta_next * Z[static_cast<size_t>(j) * steps + steps - 1]);
    lo = std::min(lo, lam[j] - r);
    up = std::max(up, lam[j] + r);
  }
  if (!std::isfinite(lo) || !std::isfinite(up) || lo > up)
    throw Error(FE_ERR_NONFINITE, "ChebyshevSolver: invalid spectral bound estimates.");
  lower_out = lo;
  upper_out = up;
}

// Device eigensolver for the projected k-by-k matrix (syevd.cu): replaces the
// reference's Dsyevd (src/gpu/CudaLanczosWorkspace.cpp:155-157) and host Eigen
// SelfAdjointEigenSolver (src/core/RitzExtraction.cpp:104).
class ProjectedEig {
 public:
  ProjectedEig(Context& ctx, int64_t cap) : ctx_(ctx), cap_(cap) {
    work_.resize(syevd_single_workspace_bytes(cap));
    info_.resize(sizeof(int));
  }
  // P (k-by-k, ldp) is overwritten by eigenvectors; W gets ascending eigenvalues.
  void run(double* P, int64_t k, int64_t ldp, double* W) {
    FE_REQUIRE(k <= cap_, "projected eigensolve larger than its capacity");
    syevd_single(P, ldp, k, W, info_.as<int32_t>(), work_.get(), work_.bytes(), ctx_.stream);
  }
  int* info() const { return info_.as<int>(); }

 private:
  Context& ctx_;
  int64_t cap_;
  DeviceBuffer work_, info_;
};

// Per-precision block set of the Chebyshev iteration.
template <typename T>
struct ChebBlocks {
  Block<T> V;   // "vectors": n x capacity
  Block<T> S;   // filter scratch, also the A*X Ritz block
  Block<T> Q;   // orthonormal basis
  Block<T> AQ;  // A*Q
  void allocate(int64_t n, int64_t cap) {
    V.allocate(n, cap);
    S.allocate(n, cap);
    Q.allocate(n, cap);
    AQ.allocate(n, cap);
  }
};

struct SmallState {
  DeviceBuffer G, Rinv, W, rel, rnorm, xnorm, info, gws, rws, cws;
  DeviceBuffer Gk, Tmp, dscale;  // fused Rayleigh-Ritz: Gram, product scratch, scaling
  int64_t cap = 0;
  bool tensor_cores = false;  // FP32 Grams/rotations on tcgen05 (3xTF32)
  int64_t precise_grams = 0;  // FP32 Cholesky passes redone with the FP64-accumulated Gram
  void allocate(int64_t n, int64_t c, bool tc) {
    cap = c;
    tensor_cores = tc;
    G.resize(static_cast<size_t>(c) * c * sizeof(double));
    Rinv.resize(static_cast<size_t>(c) * c * sizeof(double));
    Gk.resize(static_cast<size_t>(c) * c * sizeof(double));
    Tmp.resize(static_cast<size_t>(c) * c * sizeof(double));
    dscale.resize(c * sizeof(double));
    W.resize(c * sizeof(double));
    rel.resize(c * sizeof(double));
    rnorm.resize(c * sizeof(double));
    xnorm.resize(c * sizeof(double));
    info.resize(4 * sizeof(int32_t));
    size_t g = gram_workspace_bytes(n, c, c);
    if (tc) g = std::max(g, tc_gram_workspace_bytes(n, c, c));
    gws.resize(std::max<size_t>(g, 64));
    rws.resize(std::max<size_t>(residual_workspace_bytes(n, c), 64));
    if (tc) cws.resize(std::max<size_t>(tc_rotate_workspace_bytes(c, c), 64));
  }
};

inline bool tc_ok(const void* p, int64_t ld) {
  return (reinterpret_cast<uintptr_t>(p) & 15u) == 0 && ld % 4 == 0;
}

// G (ldg) = X^T Y. FP32 blocks use the tensor-core split-TF32 Gram unless
// `precise` asks for the FP64-accumulated one.
template <typename T>
void gram_block(SmallState& sm, const T* X, int64_t ldx, const T* Y, int64_t ldy, int64_t n,
                int64_t k, int64_t m, double* G, cudaStream_t s, bool precise = false) {
  if constexpr (sizeof(T) == 4) {
    if (sm.tensor_cores && !precise && ldx % 4 == 0 && ldy % 4 == 0 && n >= 128) {
      gram_tc(X, ldx, Y, ldy, n, k, m, G, sm.cap, sm.gws.get(), sm.gws.bytes(), s);
      return;
    }
    if (precise && X == Y && ldx == ldy && n >= 128) {
      // The FP64-accumulated Gram of an FP32 block: widen it once (FP32 values are
      // exact in FP64) and take the FP64 tensor-core Gram, upper tiles only.
      Block<double> wide;
      wide.allocate(n, k);
      convert<float, double>(X, ldx, wide.data(), wide.ld, n, k, s);
      gram<double>(wide.data(), wide.ld, wide.data(), wide.ld, n, k, k, G, sm.cap, sm.gws.get(),
                   sm.gws.bytes(), s);
      return;
    }
  }
  gram<T>(X, ldx, Y, ldy, n, k, m, G, sm.cap, sm.gws.get(), sm.gws.bytes(), s);
}

// Y = alpha X C + beta Y (C: FP64 column-major with leading dimension cap).
template <typename T>
void rotate_block(SmallState& sm, const T* X, int64_t ldx, const double* C, T* Y, int64_t ldy,
                  int64_t n, int64_t k, int64_t m, double alpha, double beta, cudaStream_t s,
                  bool upper_tri = false) {
  if constexpr (sizeof(T) == 4) {
    if (sm.tensor_cores && tc_ok(X, ldx) && n >= 128) {
      rotate_tc(X, ldx, C, sm.cap, Y, ldy, n, k, m, alpha, beta, sm.cws.get(), sm.cws.bytes(), s,
                upper_tri);
      return;
    }
  }
  rotate<T>(X, ldx, C, sm.cap, Y, ldy, n, k, m, alpha, beta, s, upper_tri);
}

// R^{-1} of chol(G) into Rinv, info as potrf_upper: one fused shared-memory launch for
// k <= 128; otherwise the factorization in G (which then holds R) and the inverse.
void chol_inverse(double* G, int64_t k, int64_t ldg, double* Rinv, int64_t ldi, int32_t* info,
                  cudaStream_t s) {
  if (chol_inv_small_fits(k)) {
    chol_inv_upper_batched(G, k, ldg, 0, Rinv, ldi, 0, 1, info, s);
  } else {
    potrf_upper(G, k, ldg, info, s);
    trinv_upper(G, ldg, Rinv, ldi, k, s);
  }
}

// Cholesky QR of src (n x k) into dst: G = src^T src, R = chol(G), dst = src R^{-1}
// (cuda_cholesky_qr_in_place, src/core/Orthogonalization.cpp:185-246).
// The rank-loss flag accumulates into info[slot]. With tensor-core Grams, a
// failed factorization is retried once with the FP64-accumulated Gram.
template <typename T>
void cholqr(Context& ctx, SmallState& sm, const T* src, int64_t lds, T* dst, int64_t ldd, int64_t n,
            int64_t k, int slot) {
  cudaStream_t s = ctx.stream;
  double* G = sm.G.as<double>();
  int32_t* info = sm.info.as<int32_t>() + slot;
  gram_block<T>(sm, src, lds, src, lds, n, k, k, G, s);
  chol_inverse(G, k, sm.cap, sm.Rinv.as<double>(), sm.cap, info, s);
  if (sizeof(T) == 4 && sm.tensor_cores) {
    int32_t h = 0;
    ctx.to_host(&h, info, 1);
    ctx.sync();
    if (h != 0) {
      sm.precise_grams += 1;
      gram_block<T>(sm, src, lds, src, lds, n, k, k, G, s, /*precise=*/true);
      chol_inverse(G, k, sm.cap, sm.Rinv.as<double>(), sm.cap, info, s);
    }
  }
  rotate_block<T>(sm, src, lds, sm.Rinv.as<double>(), dst, ldd, n, k, k, 1.0, 0.0, s,
                  /*upper_tri=*/true);
}

// Rayleigh-Ritz on the span of a block Y (n x k, columns independent but not
// orthonormal) as the generalized problem (Y^T A Y) c = theta (Y^T Y) c: with
// D = diag(Y^T Y)^{-1/2} and D Y^T Y D = R^T R, P = R^{-T} D (Y^T A Y) D R^{-1} = Z Theta Z^T
// and the Ritz vectors are X = Y (D R^{-1} Z). This is the reference's Cholesky QR of Y
// followed by its Rayleigh-Ritz (src/core/Orthogonalization.cpp:185-246,
// src/core/RitzExtraction.cpp:65-141) with the QR's rotation folded into the Ritz
// rotation: one n x k x k product instead of two. AY receives op*Y; P = sm.G holds Z
// and sm.W the ascending Ritz values on return. Returns false (nothing written to X)
// when the scaled Gram is not positive definite, so the caller can take the
// Cholesky QR path instead.
template <typename T>
bool fused_rr(Context& ctx, SmallState& sm, ProjectedEig& eig, const Csr& A, double sign,
              const T* Y, int64_t ldy, T* AY, int64_t lday, T* X, int64_t ldx, int64_t n, int64_t k,
              Stats& st, const double* theta = nullptr, float* y32 = nullptr,
              float* e32 = nullptr, int64_t ld32 = 0) {
  cudaStream_t s = ctx.stream;
  const int64_t ld = sm.cap;
  double* G = sm.Gk.as<double>();
  double* H = sm.G.as<double>();
  double* d = sm.dscale.as<double>();
  int32_t* info = sm.info.as<int32_t>() + 3;
  csr_spmm<T>(A, Y, ldy, AY, lday, nullptr, 0, k, sign, 0.0, 0.0, s);
  st.spmm_launches += 1;
  gram_block<T>(sm, Y, ldy, Y, ldy, n, k, k, G, s);
  bool split = false;
  if constexpr (std::is_same_v<T, double>) {
    // FP64 columns with Ritz estimates theta (the mixed path's FP64 cycles): Y^T A Y =
    // (Y^T Y) diag(theta) + Y^T E with E = AY - Y diag(theta) about a residual's size
    // against AY, so Y^T E needs only FP32-level relative accuracy (split-TF32 tensor
    // cores on FP32 copies of Y and E); Y^T Y stays an FP64 Gram.
    if (theta && y32 && e32) {
      shift_split(n, k, AY, lday, Y, ldy, theta, y32, e32, ld32, s);
      double* H1 = sm.Tmp.as<double>();
      gram_block<float>(sm, y32, ld32, e32, ld32, n, k, k, H1, s);
      gram_shift_combine(k, ld, G, theta, H1, H, s);
      split = true;
    }
  }
  if (!split) gram_block<T>(sm, Y, ldy, AY, lday, n, k, k, H, s);
  double* Rinv = sm.Rinv.as<double>();
  auto factor = [&] {
    FE_CHECK_CUDA(cudaMemsetAsync(info, 0, sizeof(int32_t), s));
    inv_sqrt_diag(G, k, ld, d, s);
    diag_scale(G, k, k, ld, d, true, s);
    chol_inverse(G, k, ld, Rinv, ld, info, s);
    int32_t h = 0;
    ctx.to_host(&h, info, 1);
    ctx.sync();
    return h == 0;
  };
  if (!factor()) {
    if (sizeof(T) == 4 && sm.tensor_cores) {
      // FP32 blocks: retry once with the FP64-accumulated Gram.
      sm.precise_grams += 1;
      gram_block<T>(sm, Y, ldy, Y, ldy, n, k, k, G, s, /*precise=*/true);
      if (!factor()) return false;
    } else {
      return false;
    }
  }
  diag_scale(H, k, k, ld, d, true, s);
  double* Tm = sm.Tmp.as<double>();
  small_gemm(false, k, k, k, 1.0, H, ld, Rinv, ld, 0.0, Tm, ld, s);    // H R^-1
  small_gemm(true, k, k, k, 1.0, Rinv, ld, Tm, ld, 0.0, H, ld, s);     // R^-T H R^-1
  symmetrize(H, k, ld, s);
  eig.run(H, k, ld, sm.W.as<double>());
  small_gemm(false, k, k, k, 1.0, Rinv, ld, H, ld, 0.0, Tm, ld, s);    // R^-1 Z
  diag_scale(Tm, k, k, ld, d, false, s);                                // D R^-1 Z
  rotate_block<T>(sm, Y, ldy, Tm, X, ldx, n, k, k, 1.0, 0.0, s);
  return true;
}

// Filter scaling (src/ChebyshevSolver.cpp:231-239) for a damped interval [cutoff, upper]
// where the amplification at `lower` is `amp` (the reference: amp = 1e3).
double reference_cutoff(double lower, double upper, int64_t degree, double amp) {
  const double xlb = std::cosh(std::acosh(amp) / static_cast<double>(degree));
  return (2.0 * lower + upper * (xlb - 1.0)) / (1.0 + xlb);
}

template <typename T>
struct ChebLoop {
  Context& ctx;
  const Csr& A;
  const Options& opt;
  SmallState& sm;
  ProjectedEig& eig;
  ChebBlocks<T> b;
  int64_t n, nev, cap, degree;
  double sign, lower, upper;
  bool cholqr2;
  bool hard;  // hard locking: the locked prefix is final, QR and Rayleigh-Ritz see the rest
  bool fused = false;  // Rayleigh-Ritz with the (second) Cholesky QR pass folded in
  // FP64 cycles of the mixed path: filter through the FP32 correction recurrence
  // (refined_filter) when every active column has a Ritz value from the last cycle.
  bool refine = false;
  bool theta_ready = false;
  Block<float> r32, z0, z1;  // refined-filter blocks (allocated on first use)
  DeviceBuffer wave_sync;    // multi-step filter's completion counters (allocated on first use)
  DeviceBuffer theta_dev;    // Ritz estimates of the columns the refined filter ran on
  bool theta_valid = false;  // set by refined_filter for the current cycle
  PhaseEvents ev;

  ChebLoop(Context& c, const Csr& a, const Options& o, SmallState& s, ProjectedEig& e, double sg,
           double lo, double up, bool two_pass)
      : ctx(c), A(a), opt(o), sm(s), eig(e), n(a.rows), nev(o.nev), degree(o.degree), sign(sg),
        lower(lo), upper(up), cholqr2(two_pass), hard(o.locking == "hard") {}

  // One filter + deflation + QR + Rayleigh-Ritz cycle (src/ChebyshevSolver.cpp:151-184).
  // On return the host holds the Ritz values W[0:sub], residuals rel[0:sub] and info.
  void iterate(int64_t locked, int64_t sub, double cutoff, std::vector<double>& W,
               std::vector<double>& rel, int32_t* info_host, Stats& st) {
    cudaStream_t s = ctx.stream;
    const int64_t active = sub - locked;
    // The filter's SpMM and the deflation's tensor-core rotation want a block that
    // starts 16-byte aligned and spans whole 16-byte vectors. When V's active
    // columns [locked, sub) do not, they are staged in S, padded with zero columns
    // to a whole number of vectors (the padding never mixes into real columns),
    // filtered and deflated there, and copied back.
    const int64_t vw = 16 / static_cast<int64_t>(sizeof(T));
    const bool in_place = locked % vw == 0 && active % vw == 0;
    const int64_t act_pad = ((active + vw - 1) / vw) * vw;
    auto stage_active = [&] {
      FE_CHECK_CUDA(cudaMemcpy2DAsync(b.S.data(), b.S.ld * sizeof(T), b.V.col(locked),
                                      b.V.ld * sizeof(T), active * sizeof(T), n,
                                      cudaMemcpyDeviceToDevice, s));
      if (act_pad > active)
        FE_CHECK_CUDA(cudaMemset2DAsync(b.S.col(active), b.S.ld * sizeof(T), 0,
                                        (act_pad - active) * sizeof(T), n, s));
    };
    FE_CHECK_CUDA(cudaMemsetAsync(sm.info.get(), 0, 4 * sizeof(int32_t), s));
    theta_valid = false;
    ev.record(0, s);
    // 1. Filter Y = T_degree(c*op + d*I) X_active, in place on V's active columns.
    if (upper != cutoff) {
      const double c = 2.0 / (upper - cutoff);
      const double d = -(upper + cutoff) / (upper - cutoff);
      if (!std::isfinite(c) || !std::isfinite(d))
        throw Error(FE_ERR_NONFINITE, "ChebyshevSolver: invalid filter scaling.");
      // The operator is sign*A: fold the sign into c.
      bool refined = false;
      if constexpr (std::is_same_v<T, double>) {
        if (refine && theta_ready) {
          std::vector<double> theta(static_cast<size_t>(act_pad), 0.0);
          for (int64_t j = 0; j < active; ++j) theta[j] = W[locked + j];
          if (in_place) {
            refined_filter(b.V.col(locked), b.V.ld, active, c, d, theta);
          } else {
            stage_active();
            refined_filter(b.S.data(), b.S.ld, act_pad, c, d, theta);
          }
          refined = true;
        }
      }
      if (!refined) {
        if (in_place) {
          filter(b.V.col(locked), b.V.ld, b.S.data(), b.S.ld, active, sign * c, d);
        } else {
          stage_active();
          filter(b.S.data(), b.S.ld, b.Q.data(), b.Q.ld, act_pad, sign * c, d);
        }
      }
      st.spmm_launches += static_cast<double>(degree);
    } else if (!in_place) {
      stage_active();
    }
    ev.record(1, s);
    // 2. Deflate against locked vectors with two-pass block Gram-Schmidt
    // (block_gram_schmidt, src/core/Orthogonalization.cpp:482-527), on the
    // aligned block (V's active columns, or their staged copy in S).
    T* Y = in_place ? b.V.col(locked) : b.S.data();
    const int64_t ldy = in_place ? b.V.ld : b.S.ld;
    if (locked > 0) {
      for (int pass = 0; pass < 2; ++pass) {
        gram_block<T>(sm, b.V.data(), b.V.ld, Y, ldy, n, locked, active, sm.G.as<double>(), s);
        rotate_block<T>(sm, b.V.data(), b.V.ld, sm.G.as<double>(), Y, ldy, n, locked, active, -1.0,
                        1.0, s);
      }
    }
    if (hard) {
      iterate_active(locked, sub, Y, ldy, W, rel, info_host, st);
      return;
    }
    if (!in_place) {
      FE_CHECK_CUDA(cudaMemcpy2DAsync(b.V.col(locked), b.V.ld * sizeof(T), b.S.data(),
                                      b.S.ld * sizeof(T), active * sizeof(T), n,
                                      cudaMemcpyDeviceToDevice, s));
    }
    // 3. Cholesky QR of the current subspace (CholQR2 on FP32 blocks).
    if (cholqr2) {
      cholqr<T>(ctx, sm, b.V.data(), b.V.ld, b.S.data(), b.S.ld, n, sub, 0);
      cholqr<T>(ctx, sm, b.S.data(), b.S.ld, b.Q.data(), b.Q.ld, n, sub, 1);
    } else {
      cholqr<T>(ctx, sm, b.V.data(), b.V.ld, b.Q.data(), b.Q.ld, n, sub, 0);
    }
    ev.record(2, s);
    // 4. Rayleigh-Ritz: AQ = op*Q, P = Q^T AQ, eig(P), rotate Q, residuals.
    csr_spmm<T>(A, b.Q.data(), b.Q.ld, b.AQ.data(), b.AQ.ld, nullptr, 0, sub, sign, 0.0, 0.0, s);
    st.spmm_launches += 1;
    double* P = sm.G.as<double>();
    gram_block<T>(sm, b.Q.data(), b.Q.ld, b.AQ.data(), b.AQ.ld, n, sub, sub, P, s);
    symmetrize(P, sub, sm.cap, s);
    eig.run(P, sub, sm.cap, sm.W.as<double>());
    rotate_block<T>(sm, b.Q.data(), b.Q.ld, P, b.V.data(), b.V.ld, n, sub, sub, 1.0, 0.0, s);
    // Residuals are read for the nev wanted pairs only (locking and the stopping
    // test), so op*V is formed for those columns by one SpMM, which moves
    // n*nev*(2+nnz/n) values where rotating AQ (the reference's AQ*P) is an
    // n x sub x sub product; it is also the true product rather than a rotated one.
    const int64_t nres = std::min(nev, sub);
    csr_spmm<T>(A, b.V.data(), b.V.ld, b.S.data(), b.S.ld, nullptr, 0, nres, sign, 0.0, 0.0, s);
    st.spmm_launches += 1;
    residual_norms<T>(b.S.data(), b.V.data(), nullptr, b.V.ld, n, nres, sm.W.as<double>(), nullptr,
                      0, sm.rnorm.as<double>(), sm.xnorm.as<double>(), sm.rel.as<double>(),
                      sm.rws.get(), sm.rws.bytes(), s, 1);
    W.resize(sub);
    rel.assign(sub, 0.0);  // guard columns: residuals not formed
    ctx.to_host(W.data(), sm.W.as<double>(), sub);
    ctx.to_host(rel.data(), sm.rel.as<double>(), nres);
    ctx.to_host(info_host, sm.info.as<int32_t>(), 2);
    ctx.to_host(info_host + 2, eig.info(), 1);
    ev.record(3, s);
    ctx.sync();
    ev.accumulate(st);
  }

  // Steps 3-4 under hard locking. The locked prefix V[:, :locked] holds final
  // Ritz vectors; the filtered block Y (active columns, deflated against the
  // prefix, 16-byte aligned: V's own columns or the staging copy in S) is
  // orthonormalized and Rayleigh-Ritz projected on its own, so the QR and the
  // projection cost n*active^2 instead of n*sub^2 once most pairs have locked. The
  // prefix's Ritz values and residuals stay as they were when they locked; only
  // W[locked:sub] and rel[locked:nev] are renewed.
  void iterate_active(int64_t locked, int64_t sub, const T* Y, int64_t ldy,
                      std::vector<double>& W, std::vector<double>& rel, int32_t* info_host,
                      Stats& st) {
    cudaStream_t s = ctx.stream;
    const int64_t active = sub - locked;
    const int64_t vw = 16 / static_cast<int64_t>(sizeof(T));
    bool done = false;
    bool ritz_in_v = false;  // the Ritz vectors were written to V[:, locked:] directly
    if (fused) {
      // FP32 blocks: one Cholesky QR pass, its second pass folded into the
      // Rayleigh-Ritz; FP64 blocks (the mixed path's FP64 cycles, whose filtered
      // columns are near-orthogonal once scaled): the Rayleigh-Ritz directly.
      const T* Yq = Y;
      int64_t ldq = ldy;
      if (cholqr2) {
        cholqr<T>(ctx, sm, Y, ldy, b.Q.data(), b.Q.ld, n, active, 0);
        Yq = b.Q.data();
        ldq = b.Q.ld;
      }
      ev.record(2, s);
      // The Ritz vectors go to S, or to Q (then copied to S) when Y is staged in S; or,
      // when the first QR pass moved the block into Q and V's active columns are
      // 16-byte aligned, straight into V[:, locked:] (no copy back afterwards).
      const bool y_in_s = Yq == b.S.data();
      ritz_in_v = Yq == b.Q.data() && aligned16(b.V.col(locked)) && b.V.ld % vw == 0;
      T* Xo = ritz_in_v ? b.V.col(locked) : (y_in_s ? b.Q.data() : b.S.data());
      const int64_t ldxo = ritz_in_v ? b.V.ld : (y_in_s ? b.Q.ld : b.S.ld);
      // FP64 cycles after a refined filter: the projected operator from the residual
      // split (fused_rr), on the refined filter's free FP32 blocks
      const bool split = std::is_same_v<T, double> && theta_valid && opt.tail_rr == "split" &&
                         z0.data() != nullptr;
      done = fused_rr<T>(ctx, sm, eig, A, sign, Yq, ldq, b.AQ.data(), b.AQ.ld, Xo, ldxo, n,
                         active, st, split ? theta_dev.as<double>() : nullptr,
                         split ? z0.data() : nullptr, split ? z1.data() : nullptr,
                         split ? z0.ld : 0);
      if (!done) ritz_in_v = false;
      if (done && y_in_s && !ritz_in_v) {
        FE_CHECK_CUDA(cudaMemcpy2DAsync(b.S.data(), b.S.ld * sizeof(T), b.Q.data(),
                                        b.Q.ld * sizeof(T), active * sizeof(T), n,
                                        cudaMemcpyDeviceToDevice, s));
      }
      if (!done && cholqr2) {  // fall back to the second Cholesky QR pass
        cholqr<T>(ctx, sm, b.Q.data(), b.Q.ld, b.AQ.data(), b.AQ.ld, n, active, 1);
        FE_CHECK_CUDA(cudaMemcpy2DAsync(b.Q.data(), b.Q.ld * sizeof(T), b.AQ.data(),
                                        b.AQ.ld * sizeof(T), active * sizeof(T), n,
                                        cudaMemcpyDeviceToDevice, s));
      } else if (!done) {
        cholqr<T>(ctx, sm, Y, ldy, b.Q.data(), b.Q.ld, n, active, 0);
      }
    } else if (cholqr2) {
      cholqr<T>(ctx, sm, Y, ldy, b.AQ.data(), b.AQ.ld, n, active, 0);
      cholqr<T>(ctx, sm, b.AQ.data(), b.AQ.ld, b.Q.data(), b.Q.ld, n, active, 1);
    } else {
      cholqr<T>(ctx, sm, Y, ldy, b.Q.data(), b.Q.ld, n, active, 0);
    }
    if (!done) {
      if (!fused) ev.record(2, s);
      csr_spmm<T>(A, b.Q.data(), b.Q.ld, b.AQ.data(), b.AQ.ld, nullptr, 0, active, sign, 0.0,
                  0.0, s);
      st.spmm_launches += 1;
      double* P = sm.G.as<double>();
      gram_block<T>(sm, b.Q.data(), b.Q.ld, b.AQ.data(), b.AQ.ld, n, active, active, P, s);
      symmetrize(P, active, sm.cap, s);
      eig.run(P, active, sm.cap, sm.W.as<double>());
      // Ritz vectors of the active block into S (aligned), residuals of its wanted
      // pairs (indices locked..nev-1), then into V[:, locked:sub].
      rotate_block<T>(sm, b.Q.data(), b.Q.ld, P, b.S.data(), b.S.ld, n, active, active, 1.0, 0.0,
                      s);
    }
    const int64_t nw = nev - locked;
    const T* Xr = ritz_in_v ? b.V.col(locked) : b.S.data();  // the Ritz vectors
    const int64_t ldr = ritz_in_v ? b.V.ld : b.S.ld;
    const int64_t room = ritz_in_v ? b.V.ld - locked : b.S.ld;
    const int64_t nw_pad = std::min(((nw + vw - 1) / vw) * vw, room);  // whole vectors
    csr_spmm<T>(A, Xr, ldr, b.AQ.data(), b.AQ.ld, nullptr, 0, nw_pad, sign, 0.0, 0.0, s);
    st.spmm_launches += 1;
    residual_norms<T>(b.AQ.data(), Xr, nullptr, ldr, n, nw, sm.W.as<double>(), nullptr, 0,
                      sm.rnorm.as<double>(), sm.xnorm.as<double>(), sm.rel.as<double>(),
                      sm.rws.get(), sm.rws.bytes(), s, 1);
    if (!ritz_in_v) {
      FE_CHECK_CUDA(cudaMemcpy2DAsync(b.V.col(locked), b.V.ld * sizeof(T), b.S.data(),
                                      b.S.ld * sizeof(T), active * sizeof(T), n,
                                      cudaMemcpyDeviceToDevice, s));
    }
    W.resize(sub);
    rel.resize(sub, 0.0);
    std::fill(rel.begin() + nev, rel.end(), 0.0);  // guard columns: residuals not formed
    ctx.to_host(W.data() + locked, sm.W.as<double>(), active);
    ctx.to_host(rel.data() + locked, sm.rel.as<double>(), nw);
    ctx.to_host(info_host, sm.info.as<int32_t>(), 2);
    ctx.to_host(info_host + 2, eig.info(), 1);
    ev.record(3, s);
    ctx.sync();
    ev.accumulate(st);
  }

  // Chebyshev filter of FP64 columns X whose Ritz values theta are known, computed to
  // FP64 accuracy with FP32 SpMMs. With L = c op + d and t_k = T_k(L(theta_j)), the
  // filtered column is y_m = T_m(L) x = t_m x + z_m where z_k = y_k - t_k x obeys
  //   z_0 = 0, z_1 = c r, z_{k+1} = 2 L z_k - z_{k-1} + 2 c t_k r,  r = (op - theta) x,
  // the three-term recurrence of the filter (src/ChebyshevSolver.cpp:243-256) with one
  // extra term. r is formed once in FP64 and rounded to FP32; for a column near an
  // eigenvector z is small against t_m x, so the FP32 rounding of the recurrence stays
  // small against z and the result carries FP64-level accuracy, where an FP32 filter of
  // x itself would carry FP32-level error relative to y.
  void refined_filter(double* X, int64_t ldx, int64_t cols, double c, double d,
                      const std::vector<double>& theta) {
    cudaStream_t s = ctx.stream;
    if (!r32.data()) {
      r32.allocate(n, b.V.ld);
      z0.allocate(n, b.V.ld);
      z1.allocate(n, b.V.ld);
    }
    const int64_t cols4 = (cols + 3) / 4 * 4;  // 16-byte rows for the FP32 steps
    const int64_t m = degree;
    std::vector<float> delta(static_cast<size_t>(std::max<int64_t>(m - 1, 1)) * cols4, 0.0f);
    std::vector<double> tm(static_cast<size_t>(cols), 1.0);
    for (int64_t j = 0; j < cols; ++j) {
      const double x = c * theta[j] + d;
      double tprev = 1.0, tcur = x;
      for (int64_t k = 1; k < m; ++k) {
        delta[static_cast<size_t>(k - 1) * cols4 + j] = static_cast<float>(2.0 * c * tcur);
        const double tn = 2.0 * x * tcur - tprev;
        tprev = tcur;
        tcur = tn;
      }
      tm[j] = tcur;
    }
    DeviceBuffer d_delta(delta.size() * sizeof(float)), d_tm(tm.size() * sizeof(double));
    if (theta_dev.bytes() < theta.size() * sizeof(double))
      theta_dev.resize(theta.size() * sizeof(double));
    DeviceBuffer& d_theta = theta_dev;
    ctx.to_device(d_delta.as<float>(), delta.data(), delta.size());
    ctx.to_device(d_tm.as<double>(), tm.data(), tm.size());
    ctx.to_device(d_theta.as<double>(), theta.data(), theta.size());
    const int64_t ld32 = r32.ld;
    if (cols4 > cols) {
      FE_CHECK_CUDA(cudaMemset2DAsync(r32.col(cols), ld32 * sizeof(float), 0,
                                      (cols4 - cols) * sizeof(float), n, s));
      FE_CHECK_CUDA(cudaMemset2DAsync(z1.col(cols), ld32 * sizeof(float), 0,
                                      (cols4 - cols) * sizeof(float), n, s));
    }
    // r = op x - theta x (FP64 product, rounded once to FP32); z_1 = c r.
    csr_spmm<double>(A, X, ldx, b.AQ.data(), b.AQ.ld, nullptr, 0, cols, sign, 0.0, 0.0, s);
    refine_start(n, cols, b.AQ.data(), b.AQ.ld, X, ldx, d_theta.as<double>(), c, r32.data(),
                 z1.data(), ld32, s);
    float* prev = z0.data();
    float* cur = z1.data();
    for (int64_t k = 1; k < m; ++k) {
      csr_spmm_corr_f32(A, cur, ld32, prev, ld32, prev, ld32, r32.data(), ld32,
                        d_delta.as<float>() + (k - 1) * cols4, cols4, 2.0 * c * sign, 2.0 * d,
                        k == 1 ? 0.0 : -1.0, s);
      std::swap(prev, cur);
    }
    refine_finish(n, cols, d_tm.as<double>(), cur, ld32, X, ldx, s);
    ctx.sync();  // the host tables are released on return
    theta_valid = true;
  }

  void filter(T* X, int64_t ldx, T* Sc, int64_t lds, int64_t cols, double c, double d) {
    cudaStream_t s = ctx.stream;
    // Several filter steps per launch where the operator allows it (cheb_filter_wave).
    if (degree >= 2) {
      const size_t need = wave_sync_bytes(n);
      if (wave_sync.bytes() < need) wave_sync.resize(need);
      if (cheb_filter_wave<T>(A, X, ldx, Sc, lds, cols, static_cast<int>(degree), c, d,
                              wave_sync.get(), wave_sync.bytes(), s))
        return;
    }
    // Y1 = c*A*Y0 + d*Y0 into scratch; Y_k = 2c*A*Y_{k-1} + 2d*Y_{k-1} - Y_{k-2} in place.
    csr_spmm<T>(A, X, ldx, Sc, lds, nullptr, 0, cols, c, d, 0.0, s);
    T* prev = X;
    int64_t ldp = ldx;
    T* cur = Sc;
    int64_t ldc = lds;
    for (int64_t k = 2; k <= degree; ++k) {
      csr_spmm<T>(A, cur, ldc, prev, ldp, prev, ldp, cols, 2.0 * c, 2.0 * d, -1.0, s);
      std::swap(prev, cur);
      std::swap(ldp, ldc);
    }
    if (cur != X) {
      FE_CHECK_CUDA(cudaMemcpy2DAsync(X, ldx * sizeof(T), cur, ldc * sizeof(T), cols * sizeof(T),
                                      n, cudaMemcpyDeviceToDevice, s));
    }
  }
};

struct SolveOut {
  std::vector<double> values, rel;
  int64_t iterations = 0;
};

// ChebyshevSolver::solve (src/ChebyshevSolver.cpp:67-221) on the device.
void chebyshev_solve(const Csr& A, const Options& opt, double* eigenvalues, double* residuals,
                     double* eigenvectors, Stats& st) {
  const int64_t n = A.rows;
  const int64_t nev = opt.nev;
  FE_REQUIRE(A.rows == A.cols, "ChebyshevSolver: matrix must be square.");
  if (n <= 0 || nev <= 0 || nev > n)
    throw Error(FE_ERR_INVALID, "ChebyshevSolver: nev must be in [1,n].");
  if (opt.which != "sr" && opt.which != "lr")
    throw Error(FE_ERR_INVALID, "ChebyshevSolver: only SR and LR are supported.");
  FE_REQUIRE(opt.degree >= 1, "ChebyshevSolver: degree must be >= 1.");
  FE_REQUIRE(opt.precision == "fp64" || opt.precision == "mixed",
             "precision must be fp64 or mixed");
  FE_REQUIRE(opt.bounds == "reference" || opt.bounds == "ritz", "bounds must be reference or ritz");
  FE_REQUIRE(opt.init == "host" || opt.init == "device", "init must be host or device");
  const bool flip = opt.which == "lr";
  const double sign = flip ? -1.0 : 1.0;
  const unsigned seed = opt.seed_or_default();
  int64_t cap = nev + std::min(nev, n - nev);
  if (opt.block > 0) cap = std::max(nev, std::min(opt.block, n));
  const bool host_init = opt.init == "host";
  const bool mixed = opt.precision == "mixed";
  const bool fused_rr_on = opt.rr.empty() ? mixed : opt.rr == "fused";
  const bool refine_on = mixed && opt.tail_filter == "refined";

  using clock = std::chrono::steady_clock;
  const auto t_start = clock::now();
  auto ms_since = [](clock::time_point t) {
    return std::chrono::duration<double, std::milli>(clock::now() - t).count();
  };
  Context ctx;
  if (opt.verbosity >= 2)
    std::fprintf(stderr, "[fe] context %.1f ms\n", ms_since(t_start));
  SmallState sm;
  sm.allocate(n, cap, mixed && opt.tensor_cores && tc_gemm_available());
  ProjectedEig eig(ctx, cap);

  double lower = 0, upper = 0;
  const auto t_bounds = clock::now();
  lanczos_bounds(ctx, A, sign, seed, host_init, lower, upper);
  st.lower = lower;
  st.upper = upper;
  if (opt.verbosity >= 2)
    std::fprintf(stderr, "[fe] Lanczos bounds %.1f ms\n", ms_since(t_bounds));

  std::unique_ptr<ChebLoop<float>> l32;
  std::unique_ptr<ChebLoop<double>> l64;
  // Initial block and its Cholesky QR (src/ChebyshevSolver.cpp:94-107).
  {
    FE_CHECK_CUDA(cudaMemsetAsync(sm.info.get(), 0, 4 * sizeof(int32_t), ctx.stream));
    Block<double> V0;
    V0.allocate(n, cap);
    if (host_init) random_block_host<double>(ctx, V0, cap, seed);
    else fill_uniform<double>(V0.data(), V0.ld, n, cap, seed, ctx.stream);
    if (mixed) {
      l32.reset(new ChebLoop<float>(ctx, A, opt, sm, eig, sign, lower, upper, true));
      l32->fused = fused_rr_on;
      l32->b.allocate(n, cap);
      // A random block is well conditioned: round it to FP32 and orthonormalize
      // with CholQR2 on the FP32 (tensor-core) path.
      convert<double, float>(V0.data(), V0.ld, l32->b.S.data(), l32->b.S.ld, n, cap, ctx.stream);
      V0.buf.release();
      cholqr<float>(ctx, sm, l32->b.S.data(), l32->b.S.ld, l32->b.Q.data(), l32->b.Q.ld, n, cap, 0);
      cholqr<float>(ctx, sm, l32->b.Q.data(), l32->b.Q.ld, l32->b.V.data(), l32->b.V.ld, n, cap, 1);
    } else {
      l64.reset(new ChebLoop<double>(ctx, A, opt, sm, eig, sign, lower, upper, false));
      l64->fused = fused_rr_on;
      l64->b.allocate(n, cap);
      cholqr<double>(ctx, sm, V0.data(), V0.ld, l64->b.V.data(), l64->b.V.ld, n, cap, 0);
    }
    int32_t info[2] = {0, 0};
    ctx.to_host(info, sm.info.as<int32_t>(), 2);
    ctx.sync();
    if (info[0] != 0 || info[1] != 0)
      throw Error(FE_ERR_NOT_SPD, "ChebyshevSolver: initial Cholesky QR failed.");
  }
  if (opt.verbosity >= 2)
    std::fprintf(stderr, "[fe] setup (buffers, bounds, initial QR) %.1f ms\n", ms_since(t_start));

  int64_t locked = 0;
  int64_t sub = nev;
  int64_t sub_prev = 0;
  std::vector<double> W, rel, worst_history;
  int64_t it_done = 0;
  const double tol = opt.tol;
  const auto t_loop = clock::now();
  for (int64_t iter = 0; iter < opt.maxiter; ++iter) {
    // Damped interval [cutoff, upper]: the reference fixes the cutoff where the
    // filter amplifies `lower` by 1e3. bounds=ritz (after the first cycle) damps
    // from the largest Ritz value of the last Rayleigh-Ritz instead, lowered if
    // needed so that the amplification at `lower` stays within the cap.
    // The interval is set by the configured degree in every phase: a different
    // degree for the FP64 cycles (tail_degree) changes how strongly the same
    // interval is filtered, not where it lies.
    const int64_t deg_now = l32 ? opt.degree : (l64 ? l64->degree : opt.degree);
    double cutoff = reference_cutoff(lower, upper, opt.degree, 1.0e3);
    if (opt.bounds == "ritz" && sub_prev > 0) {
      cutoff = std::min(W[sub_prev - 1],
                        reference_cutoff(lower, upper, opt.degree, opt.amplification));
    }
    if (upper == lower) cutoff = upper;  // collapsed spectrum: no filtering
    int32_t info[3] = {0, 0, 0};
    const auto t_cycle = clock::now();
    if (l32) {
      l32->iterate(locked, sub, cutoff, W, rel, info, st);
      st.fp32_iterations += 1;
    } else {
      l64->theta_ready = sub_prev >= sub;  // every active column has a Ritz value
      l64->iterate(locked, sub, cutoff, W, rel, info, st);
      st.fp64_iterations += 1;
    }
    if (info[0] != 0 || info[1] != 0)
      throw Error(FE_ERR_NOT_SPD, "ChebyshevSolver: Cholesky QR failed during filtering.");
    if (info[2] != 0) throw Error(FE_ERR_CUDA, "ChebyshevSolver: projected eigensolve failed.");
    for (int64_t j = 0; j < sub; ++j)
      if (!std::isfinite(W[j]) || !std::isfinite(rel[j]))
        throw Error(FE_ERR_NONFINITE, "ChebyshevSolver: non-finite Ritz values or residuals.");
    sub_prev = sub;
    // 4. Ordered locking (src/ChebyshevSolver.cpp:186-192). On FP32 blocks, whose
    // residuals cannot reach tol, pairs lock at the FP32 floor (mixed_switch) so
    // the spare columns still enter the subspace as the prefix converges.
    const double lock_tol = l32 ? std::max(tol, opt.mixed_switch) : tol;
    if (opt.locking != "hard") locked = 0;  // soft: recheck the whole prefix (reference)
    while (locked < nev && rel[locked] <= lock_tol) ++locked;
    sub = std::max(sub, nev + std::min(locked, cap - nev));
    // FP64 cycles of the mixed path with tail_guard: the subspace keeps that many
    // columns past nev (the FP32 phase has brought every wanted pair to its floor).
    if (l64 && opt.tail_guard > 0) sub = std::min(sub, nev + opt.tail_guard);
    it_done = iter + 1;
    double worst = 0.0;
    for (int64_t j = 0; j < nev; ++j) worst = std::max(worst, rel[j]);
    if (opt.verbosity >= 2) {
      std::fprintf(stderr,
                   "[fe] iter %lld %s deg %lld sub %lld locked %lld worst %.3e cutoff %.6g "
                   "%.2f ms\n",
                   static_cast<long long>(iter + 1), l32 ? "fp32" : "fp64",
                   static_cast<long long>(deg_now), static_cast<long long>(sub_prev),
                   static_cast<long long>(locked), worst, cutoff, ms_since(t_cycle));
    }
    if (worst <= tol) break;
    worst_history.push_back(worst);
    const size_t h = worst_history.size();
    // Leave FP32 at its residual floor, or when the FP32 cycles stop reducing the
    // worst residual (no 30% gain over three cycles).
    const bool stalled = h >= 4 && worst > 0.7 * worst_history[h - 4];
    if (l32 && (worst <= std::max(opt.mixed_switch, tol) || stalled)) {
      worst_history.clear();
      const auto t_switch = clock::now();
      // FP32 residual floor reached: continue on FP64 blocks.
      l64.reset(new ChebLoop<double>(ctx, A, opt, sm, eig, sign, lower, upper, false));
      l64->fused = fused_rr_on;
      l64->refine = refine_on;
      if (opt.tail_degree > 0) l64->degree = opt.tail_degree;
      l64->b.allocate(n, cap);
      convert<float, double>(l32->b.V.data(), l32->b.V.ld, l64->b.V.data(), l64->b.V.ld, n, cap,
                             ctx.stream);
      ctx.sync();
      l32.reset();
      if (opt.verbosity >= 2)
        std::fprintf(stderr, "[fe] FP32 -> FP64 switch %.1f ms\n", ms_since(t_switch));
      locked = 0;  // FP64 sweeps refine every pair to tol
      while (locked < nev && rel[locked] <= tol) ++locked;
      if (opt.tail_guard > 0) sub = std::min(sub, nev + opt.tail_guard);
    }
  }
  // Results: eigenvalues (sign restored) and the FP64 residual check of the
  // returned vectors on the device: ||A x - l x|| / ((1 + |l|) ||x||), which
  // fasteig_problem::solve recomputes for non-Krylov solvers on the host
  // (src/fasteig_problem.cpp:419-422, src/fasteig_solver.cpp:89-129).
  // Hard locking can leave a locked pair above a Ritz value found later (an
  // eigenvalue that entered the subspace after the prefix locked); such pairs are
  // returned in ascending order, as the reference's whole-subspace Rayleigh-Ritz
  // returns them.
  std::vector<int32_t> order;
  if (opt.locking == "hard" && !std::is_sorted(W.begin(), W.begin() + nev)) {
    order.resize(nev);
    for (int64_t j = 0; j < nev; ++j) order[j] = static_cast<int32_t>(j);
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return W[a] < W[b]; });
    std::vector<double> Ws(nev);
    for (int64_t j = 0; j < nev; ++j) Ws[j] = W[order[j]];
    std::copy(Ws.begin(), Ws.end(), W.begin());
  }
  for (int64_t j = 0; j < nev; ++j) eigenvalues[j] = sign * W[j];
  if (opt.verbosity >= 2)
    std::fprintf(stderr, "[fe] filter cycles (wall) %.1f ms\n", ms_since(t_loop));
  const auto t_finish = clock::now();
  {
    cudaStream_t s = ctx.stream;
    Block<double> Xf, AXf;
    const double* Xp = nullptr;
    int64_t ldx = 0;
    if (l64) {
      Xp = l64->b.V.data();
      ldx = l64->b.V.ld;
    } else {
      Xf.allocate(n, cap);
      convert<float, double>(l32->b.V.data(), l32->b.V.ld, Xf.data(), Xf.ld, n, nev, s);
      Xp = Xf.data();
      ldx = Xf.ld;
    }
    Block<double> Xs;
    if (!order.empty()) {
      Xs.allocate(n, cap);
      DeviceBuffer idx(static_cast<size_t>(nev) * sizeof(int32_t));
      ctx.to_device(idx.as<int32_t>(), order.data(), nev);
      gather_columns<double>(Xp, ldx, idx.as<int32_t>(), nev, Xs.data(), Xs.ld, n, s);
      ctx.sync();
      Xp = Xs.data();
      ldx = Xs.ld;
    }
    AXf.allocate(n, cap);  // same leading dimension as the vector block
    csr_spmm<double>(A, Xp, ldx, AXf.data(), AXf.ld, nullptr, 0, nev, 1.0, 0.0, 0.0, s);
    ctx.to_device(sm.W.as<double>(), eigenvalues, nev);
    residual_norms<double>(AXf.data(), Xp, nullptr, ldx, n, nev, sm.W.as<double>(), nullptr, 0,
                           sm.rnorm.as<double>(), sm.xnorm.as<double>(), sm.rel.as<double>(),
                           sm.rws.get(), sm.rws.bytes(), s, 1);
    ctx.to_host(residuals, sm.rel.as<double>(), nev);
    if (eigenvectors) {
      // Row-major device block -> column-major n x nev (the copy_to_host boundary),
      // transposed on the device and copied straight into the caller's buffer.
      AXf.buf.release();
      DeviceBuffer cm(static_cast<size_t>(n) * nev * sizeof(double));
      to_colmajor(Xp, ldx, n, nev, cm.as<double>(), s);
      FE_CHECK_CUDA(cudaMemcpyAsync(eigenvectors, cm.get(), cm.bytes(), cudaMemcpyDeviceToHost, s));
      ctx.sync();
    }
    ctx.sync();
  }
  if (opt.verbosity >= 2)
    std::fprintf(stderr, "[fe] finish (FP64 residual check%s) %.1f ms\n",
                 eigenvectors ? ", vectors to host" : "", ms_since(t_finish));
  st.iterations = static_cast<double>(it_done);
  st.precise_grams = static_cast<double>(sm.precise_grams);
}

// ===========================================================================
// Shared pieces of the block solvers (LOBPCG, Davidson) on FP64 blocks.
// ===========================================================================

// Relative residuals of the returned pairs, recomputed in FP64 on the device
// (fasteig_problem::solve recomputes them for non-Krylov solvers,
// src/fasteig_problem.cpp:419-422 -> src/fasteig_solver.cpp:89-129), and the
// vectors to the host as column-major n x nev (transposed on the device).
void finish_results(Context& ctx, SmallState& sm, const Csr& A, const Csr* B, const double* X,
                    int64_t ldx, int64_t n, int64_t nev, const double* eigenvalues,
                    double* residuals, double* eigenvectors) {
  cudaStream_t s = ctx.stream;
  Block<double> AX, BX;
  AX.allocate(n, ldx);
  csr_spmm<double>(A, X, ldx, AX.data(), AX.ld, nullptr, 0, nev, 1.0, 0.0, 0.0, s);
  const double* MX = nullptr;
  if (B) {
    BX.allocate(n, ldx);
    csr_spmm<double>(*B, X, ldx, BX.data(), BX.ld, nullptr, 0, nev, 1.0, 0.0, 0.0, s);
    MX = BX.data();
  }
  FE_REQUIRE(AX.ld == ldx, "finish_results: leading dimension mismatch");
  ctx.to_device(sm.W.as<double>(), eigenvalues, nev);
  residual_norms<double>(AX.data(), X, MX, ldx, n, nev, sm.W.as<double>(), nullptr, 0,
                         sm.rnorm.as<double>(), sm.xnorm.as<double>(), sm.rel.as<double>(),
                         sm.rws.get(), sm.rws.bytes(), s, 1);
  ctx.to_host(residuals, sm.rel.as<double>(), nev);
  if (eigenvectors) {
    DeviceBuffer cm(static_cast<size_t>(n) * nev * sizeof(double));
    to_colmajor(X, ldx, n, nev, cm.as<double>(), s);
    FE_CHECK_CUDA(cudaMemcpyAsync(eigenvectors, cm.get(), cm.bytes(), cudaMemcpyDeviceToHost, s));
    ctx.sync();
  }
  ctx.sync();
}

// Reference selection order (lanczos_select_ritz_indices,
// src/core/RitzExtraction.cpp:162-179; sort_indices, include/fasteig_solver.hpp:58-82).
std::vector<int32_t> select_indices(const std::vector<double>& w, const std::string& which) {
  return ritz_order(w, which);
}

// Device Rayleigh-Ritz (extract_projected_ritz_pairs, src/core/RitzExtraction.cpp:65-141):
// P (cols x cols, ld sm.cap, device) is destroyed. X = B C, AX = AB C, R = AX - X diag(l),
// rel = ||r|| / ((1 + |l|) ||x||). C (cols x req, ld sm.cap) is left in `coef`.
struct RitzResult {
  std::vector<double> values, rel;
};

template <typename T>
void ritz_extract(Context& ctx, SmallState& sm, ProjectedEig& eig, double* P, const T* Bm,
                  const T* ABm, int64_t ld, int64_t n, int64_t cols, int64_t req,
                  const std::string& which, T* X, T* AX, T* R, double* coef,
                  DeviceBuffer& idx_dev, RitzResult& out, const T* BBm = nullptr,
                  T* BX = nullptr) {
  cudaStream_t s = ctx.stream;
  symmetrize(P, cols, sm.cap, s);
  eig.run(P, cols, sm.cap, sm.W.as<double>());
  std::vector<double> w(cols);
  int info = 0;
  ctx.to_host(w.data(), sm.W.as<double>(), cols);
  ctx.to_host(&info, eig.info(), 1);
  ctx.sync();
  if (info != 0) throw Error(FE_ERR_CUDA, "projected eigensolve failed.");
  const std::vector<int32_t> idx = select_indices(w, which);
  std::vector<int32_t> sel(idx.begin(), idx.begin() + req);
  out.values.resize(req);
  for (int64_t j = 0; j < req; ++j) out.values[j] = w[sel[j]];
  idx_dev.resize(std::max<size_t>(sel.size() * sizeof(int32_t), 4));
  ctx.to_device(idx_dev.as<int32_t>(), sel.data(), sel.size());
  small_gather_scale(P, sm.cap, cols, idx_dev.as<int32_t>(), nullptr, req, coef, sm.cap, s);
  rotate_block<T>(sm, Bm, ld, coef, X, ld, n, cols, req, 1.0, 0.0, s);
  rotate_block<T>(sm, ABm, ld, coef, AX, ld, n, cols, req, 1.0, 0.0, s);
  if (BBm) rotate_block<T>(sm, BBm, ld, coef, BX, ld, n, cols, req, 1.0, 0.0, s);
  ctx.to_device(sm.W.as<double>(), out.values.data(), req);
  residual_norms<T>(AX, X, BBm ? BX : nullptr, ld, n, req, sm.W.as<double>(), R, R ? ld : 0,
                         sm.rnorm.as<double>(), sm.xnorm.as<double>(), sm.rel.as<double>(),
                         sm.rws.get(), sm.rws.bytes(), s, 1);
  out.rel.resize(req);
  ctx.to_host(out.rel.data(), sm.rel.as<double>(), req);
  ctx.sync();
  for (int64_t j = 0; j < req; ++j)
    if (!std::isfinite(out.values[j]) || !std::isfinite(out.rel[j]))
      throw Error(FE_ERR_NONFINITE, "non-finite Ritz values or residuals.");
}

// Two-pass block Gram-Schmidt of src (n x b) against V[:, :k] into dst
// (block_gram_schmidt, src/core/Orthogonalization.cpp:482-527). dst may be src.
void block_gs(Context& ctx, SmallState& sm, const double* V, int64_t ld, int64_t k,
              const double* src, double* dst, int64_t n, int64_t b) {
  cudaStream_t s = ctx.stream;
  if (dst != src)
    FE_CHECK_CUDA(cudaMemcpy2DAsync(dst, ld * sizeof(double), src, ld * sizeof(double),
                                    b * sizeof(double), n, cudaMemcpyDeviceToDevice, s));
  if (k == 0) return;
  for (int pass = 0; pass < 2; ++pass) {
    gram_block<double>(sm, V, ld, dst, ld, n, k, b, sm.G.as<double>(), s);
    rotate_block<double>(sm, V, ld, sm.G.as<double>(), dst, ld, n, k, b, -1.0, 1.0, s);
  }
}

// Orthonormal basis of the part of `src` outside V[:, :k], dropping numerically
// dependent directions (orthonormalize_block, src/core/Orthogonalization.cpp:717-775).
// Two passes of: column norms -> block Gram-Schmidt -> Gram -> eigen-decomposition
// -> keep singular values above rank_tol * (largest column norm) -> rotate by
// U Sigma^-1. The reference takes the SVD of the Householder R of the projected
// block; the singular values and retained span are the same, computed here from the
// FP64 Gram, which resolves singular values down to ~1e-8 of the largest, so
// directions below that (and below rank_tol) are dropped. Returns the rank; the
// result is in out[:, :rank].
int64_t ortho_block(Context& ctx, SmallState& sm, ProjectedEig& eig, const double* V, int64_t ld,
                    int64_t k, const double* src, int64_t b, double* out, double* tmp,
                    int64_t n, DeviceBuffer& idx_dev, double rank_tol = 1e-12) {
  cudaStream_t s = ctx.stream;
  if (k >= n) return 0;
  const double* cur = src;
  int64_t cols = b;
  int64_t rank = 0;
  std::vector<double> norms, w, scale_v;
  for (int pass = 0; pass < 2; ++pass) {
    norms.resize(cols);
    residual_norms<double>(nullptr, cur, nullptr, ld, n, cols, nullptr, nullptr, 0, nullptr,
                           sm.xnorm.as<double>(), nullptr, sm.rws.get(), sm.rws.bytes(), s, 0);
    ctx.to_host(norms.data(), sm.xnorm.as<double>(), cols);
    ctx.sync();
    double scale = 0.0;
    for (double v : norms) {
      if (!std::isfinite(v)) throw Error(FE_ERR_NONFINITE, "orthonormalize_block: non-finite column norms.");
      scale = std::max(scale, v);
    }
    if (scale == 0.0) return 0;
    block_gs(ctx, sm, V, ld, k, cur, tmp, n, cols);
    double* G = sm.G.as<double>();
    gram_block<double>(sm, tmp, ld, tmp, ld, n, cols, cols, G, s);
    symmetrize(G, cols, sm.cap, s);
    eig.run(G, cols, sm.cap, sm.W.as<double>());
    w.resize(cols);
    ctx.to_host(w.data(), sm.W.as<double>(), cols);
    ctx.sync();
    const double smax = std::sqrt(std::max(w[cols - 1], 0.0));
    const int64_t capacity = std::min<int64_t>(cols, n - k);
    const double cut = std::max(rank_tol * scale, 1e-7 * smax);
    std::vector<int32_t> sel;
    scale_v.clear();
    for (int64_t i = cols - 1; i >= 0 && static_cast<int64_t>(sel.size()) < capacity; --i) {
      const double sv = std::sqrt(std::max(w[i], 0.0));
      if (!(sv > cut)) break;
      sel.push_back(static_cast<int32_t>(i));
      scale_v.push_back(1.0 / sv);
    }
    rank = static_cast<int64_t>(sel.size());
    if (rank == 0) return 0;
    const size_t dbl_off = ((rank * sizeof(int32_t) + 7) / 8) * 8;
    idx_dev.resize(dbl_off + rank * sizeof(double));
    int32_t* di = idx_dev.as<int32_t>();
    double* ds = reinterpret_cast<double*>(idx_dev.as<uint8_t>() + dbl_off);
    ctx.to_device(di, sel.data(), rank);
    ctx.to_device(ds, scale_v.data(), rank);
    small_gather_scale(G, sm.cap, cols, di, ds, rank, sm.Rinv.as<double>(), sm.cap, s);
    rotate_block<double>(sm, tmp, ld, sm.Rinv.as<double>(), out, ld, n, cols, rank, 1.0, 0.0, s);
    cur = out;
    cols = rank;
    ctx.sync();
  }
  return rank;
}

// Cholesky QR twice in place through `tmp` (stands in for the reference's
// Householder QR of nearly orthonormal blocks: same span, orthonormal to FP64).
void cholqr2_inplace(Context& ctx, SmallState& sm, double* X, double* tmp, int64_t ld, int64_t n,
                     int64_t b, const char* what) {
  FE_CHECK_CUDA(cudaMemsetAsync(sm.info.get(), 0, 4 * sizeof(int32_t), ctx.stream));
  cholqr<double>(ctx, sm, X, ld, tmp, ld, n, b, 0);
  cholqr<double>(ctx, sm, tmp, ld, X, ld, n, b, 1);
  int32_t info[2] = {0, 0};
  ctx.to_host(info, sm.info.as<int32_t>(), 2);
  ctx.sync();
  if (info[0] != 0 || info[1] != 0) throw Error(FE_ERR_NOT_SPD, std::string(what) + ": QR failed.");
}

void fill_initial_block(Context& ctx, double* X, int64_t ld, int64_t n, int64_t cols, unsigned seed,
                        bool host_init) {
  if (host_init) {
    std::mt19937 rng(seed);
    std::uniform_real_distribution<double> dist(-1.0, 1.0);
    std::vector<double> host(static_cast<size_t>(n) * ld, 0.0);
    for (int64_t j = 0; j < cols; ++j)
      for (int64_t i = 0; i < n; ++i) host[static_cast<size_t>(i) * ld + j] = dist(rng);
    ctx.to_device(X, host.data(), host.size());
    ctx.sync();
  } else {
    fill_uniform<double>(X, ld, n, cols, seed, ctx.stream);
  }
}

// LOBPCGSolver::solve (src/LOBPCGSolver.cpp:25-174): unpreconditioned LOBPCG with
// block width nev, soft locking, basis [X W P] of at most min(n, 3 nev) columns.
void lobpcg_solve(const Csr& A, const Options& opt, double* eigenvalues, double* residuals,
                  double* eigenvectors, Stats& st) {
  const int64_t n = A.rows, nev = opt.nev;
  if (n <= 0 || nev <= 0 || nev > n || opt.maxiter <= 0)
    throw Error(FE_ERR_INVALID, "LOBPCGSolver: require 0 < nev <= n and maxiter > 0.");
  if (opt.which != "sr" && opt.which != "lr")
    throw Error(FE_ERR_INVALID, "LOBPCGSolver: only SR and LR are supported.");
  const double sign = opt.which == "lr" ? -1.0 : 1.0;
  const double tol = opt.tol;
  const int64_t cap = std::min<int64_t>(n, 3 * nev);
  Context ctx;
  cudaStream_t s = ctx.stream;
  SmallState sm;
  sm.allocate(n, cap, false);
  ProjectedEig eig(ctx, cap);
  Block<double> X, AX, R, Pd, S, AS, T1, T2, Wsrc;
  for (Block<double>* b : {&X, &AX, &R, &Pd, &S, &AS, &T1, &T2, &Wsrc}) b->allocate(n, cap);
  const int64_t ld = X.ld;
  DeviceBuffer idx_dev(static_cast<size_t>(cap) * 16), coef(static_cast<size_t>(cap) * cap * sizeof(double));
  fill_initial_block(ctx, X.data(), ld, n, nev, opt.seed_or_default(), opt.init == "host");
  cholqr2_inplace(ctx, sm, X.data(), T1.data(), ld, n, nev, "LOBPCGSolver: initial");
  csr_spmm<double>(A, X.data(), ld, AX.data(), ld, nullptr, 0, nev, sign, 0.0, 0.0, s);
  st.spmm_launches += 1;
  // Rayleigh-Ritz on span(X) (src/LOBPCGSolver.cpp:72-78).
  FE_CHECK_CUDA(cudaMemcpy2DAsync(S.data(), ld * 8, X.data(), ld * 8, nev * 8, n,
                                  cudaMemcpyDeviceToDevice, s));
  FE_CHECK_CUDA(cudaMemcpy2DAsync(AS.data(), ld * 8, AX.data(), ld * 8, nev * 8, n,
                                  cudaMemcpyDeviceToDevice, s));
  gram_block<double>(sm, S.data(), ld, AS.data(), ld, n, nev, nev, sm.G.as<double>(), s);
  RitzResult ritz;
  ritz_extract(ctx, sm, eig, sm.G.as<double>(), S.data(), AS.data(), ld, n, nev, nev, "sr",
               X.data(), AX.data(), R.data(), coef.as<double>(), idx_dev, ritz);
  bool have_p = false;
  int64_t it_done = 0;
  for (int64_t iter = 0; iter < opt.maxiter; ++iter) {
    double worst = 0;
    for (double v : ritz.rel) worst = std::max(worst, v);
    if (worst <= tol) break;
    std::vector<int32_t> active;
    for (int64_t j = 0; j < nev; ++j)
      if (ritz.rel[j] > tol) active.push_back(static_cast<int32_t>(j));
    const int64_t na = static_cast<int64_t>(active.size());
    DeviceBuffer act(na * sizeof(int32_t));
    ctx.to_device(act.as<int32_t>(), active.data(), na);
    gather_columns<double>(R.data(), ld, act.as<int32_t>(), na, Wsrc.data(), ld, n, s);
    cholqr2_inplace(ctx, sm, X.data(), T1.data(), ld, n, nev, "LOBPCGSolver: Ritz-vector");
    FE_CHECK_CUDA(cudaMemcpy2DAsync(S.data(), ld * 8, X.data(), ld * 8, nev * 8, n,
                                    cudaMemcpyDeviceToDevice, s));
    int64_t cols = nev;
    const int64_t rw = ortho_block(ctx, sm, eig, S.data(), ld, cols, Wsrc.data(), na, T1.data(),
                                   T2.data(), n, idx_dev);
    if (rw > 0) {
      FE_CHECK_CUDA(cudaMemcpy2DAsync(S.col(cols), ld * 8, T1.data(), ld * 8, rw * 8, n,
                                      cudaMemcpyDeviceToDevice, s));
      cols += rw;
    }
    if (have_p && cols < cap) {
      gather_columns<double>(Pd.data(), ld, act.as<int32_t>(), na, Wsrc.data(), ld, n, s);
      int64_t rp = ortho_block(ctx, sm, eig, S.data(), ld, cols, Wsrc.data(), na, T1.data(),
                               T2.data(), n, idx_dev);
      rp = std::min(rp, cap - cols);
      if (rp > 0) {
        FE_CHECK_CUDA(cudaMemcpy2DAsync(S.col(cols), ld * 8, T1.data(), ld * 8, rp * 8, n,
                                        cudaMemcpyDeviceToDevice, s));
        cols += rp;
      }
    }
    // Rayleigh-Ritz in S = [X W P] with a fresh A*S (src/LOBPCGSolver.cpp:134-138).
    csr_spmm<double>(A, S.data(), ld, AS.data(), ld, nullptr, 0, cols, sign, 0.0, 0.0, s);
    st.spmm_launches += 1;
    gram_block<double>(sm, S.data(), ld, AS.data(), ld, n, cols, cols, sm.G.as<double>(), s);
    ritz_extract(ctx, sm, eig, sm.G.as<double>(), S.data(), AS.data(), ld, n, cols, nev, "sr",
                 X.data(), AX.data(), R.data(), coef.as<double>(), idx_dev, ritz);
    // P = S C with the X rows of C zeroed (src/LOBPCGSolver.cpp:147-150).
    FE_CHECK_CUDA(cudaMemset2DAsync(coef.get(), cap * 8, 0, nev * 8, nev, s));
    rotate_block<double>(sm, S.data(), ld, coef.as<double>(), Pd.data(), ld, n, cols, nev, 1.0, 0.0,
                         s);
    have_p = true;
    it_done = iter + 1;
    worst = 0;
    for (double v : ritz.rel) worst = std::max(worst, v);
    if (opt.verbosity >= 2)
      std::fprintf(stderr, "[fe] lobpcg iter %lld cols %lld worst %.3e\n",
                   static_cast<long long>(iter + 1), static_cast<long long>(cols), worst);
    if (worst <= tol || cols == nev) break;
  }
  for (int64_t j = 0; j < nev; ++j) eigenvalues[j] = sign * ritz.values[j];
  finish_results(ctx, sm, A, nullptr, X.data(), ld, n, nev, eigenvalues, residuals, eigenvectors);
  st.iterations = static_cast<double>(it_done);
  st.fp64_iterations = static_cast<double>(it_done);
}

// DavidsonSolver::solve (src/DavidsonSolver.cpp:27-264): block Davidson with thick
// restart, unpreconditioned residual corrections, locktol = min(1e-5, tol).
void davidson_solve(const Csr& A, const Options& opt, double* eigenvalues, double* residuals,
                    double* eigenvectors, Stats& st) {
  const int64_t n = A.rows, nev = opt.nev;
  if (n <= 0) throw Error(FE_ERR_INVALID, "DavidsonSolver: n must be > 0.");
  if (nev <= 0 || nev > n) throw Error(FE_ERR_INVALID, "DavidsonSolver: nev must be in [1,n].");
  if (opt.maxiter <= 0) throw Error(FE_ERR_INVALID, "DavidsonSolver: maxiter must be > 0.");
  if (opt.maxblks < 1) throw Error(FE_ERR_INVALID, "DavidsonSolver: maxblks must be at least 1.");
  const std::string which = opt.which;
  if (which == "sai")
    throw Error(FE_ERR_INVALID, "DavidsonSolver: SAI is not supported yet; use SR/LR/SM/LM/BE.");
  if (which != "sr" && which != "lr" && which != "sm" && which != "lm" && which != "be")
    throw Error(FE_ERR_INVALID, "DavidsonSolver: invalid which option (use SR/LR/SM/LM/BE).");
  const double tol = opt.tol;
  const int64_t cap = std::min<int64_t>(n, opt.maxblks * nev);
  Context ctx;
  cudaStream_t s = ctx.stream;
  SmallState sm;
  sm.allocate(n, cap, false);
  ProjectedEig eig(ctx, cap);
  Block<double> V, AV, X, AX, R, Cb, ACb, T1;
  for (Block<double>* b : {&V, &AV, &X, &AX, &R, &Cb, &ACb, &T1}) b->allocate(n, cap);
  const int64_t ld = V.ld;
  DeviceBuffer idx_dev(static_cast<size_t>(cap) * 16), coef(static_cast<size_t>(cap) * cap * sizeof(double));
  DeviceBuffer proj(static_cast<size_t>(cap) * cap * sizeof(double));
  double* Pm = proj.as<double>();
  double* Pw = sm.G.as<double>();
  auto extract = [&](int64_t cols, RitzResult& out) {
    FE_CHECK_CUDA(cudaMemcpy2DAsync(Pw, cap * 8, Pm, cap * 8, cols * 8, cols,
                                    cudaMemcpyDeviceToDevice, s));
    ritz_extract(ctx, sm, eig, Pw, V.data(), AV.data(), ld, n, cols, nev, which, X.data(),
                 AX.data(), R.data(), coef.as<double>(), idx_dev, out);
  };
  // Initial block: random, Cholesky QR (src/DavidsonSolver.cpp:59-79).
  fill_initial_block(ctx, X.data(), ld, n, nev, opt.seed_or_default(), opt.init == "host");
  {
    FE_CHECK_CUDA(cudaMemsetAsync(sm.info.get(), 0, 4 * sizeof(int32_t), s));
    cholqr<double>(ctx, sm, X.data(), ld, V.data(), ld, n, nev, 0);
    int32_t info = 0;
    ctx.to_host(&info, sm.info.as<int32_t>(), 1);
    ctx.sync();
    if (info != 0) throw Error(FE_ERR_NOT_SPD, "DavidsonSolver: initial Cholesky QR failed.");
  }
  csr_spmm<double>(A, V.data(), ld, AV.data(), ld, nullptr, 0, nev, 1.0, 0.0, 0.0, s);
  st.spmm_launches += 1;
  gram_block<double>(sm, V.data(), ld, AV.data(), ld, n, nev, nev, Pm, s);
  RitzResult ritz;
  extract(nev, ritz);
  const double locktol = std::min(1.0e-5, tol);
  int64_t it_done = 0;
  for (int64_t iter = 0; iter < opt.maxiter; ++iter) {
    // Thick restart (src/DavidsonSolver.cpp:131-155).
    cholqr2_inplace(ctx, sm, X.data(), T1.data(), ld, n, nev, "DavidsonSolver: restart");
    FE_CHECK_CUDA(cudaMemcpy2DAsync(V.data(), ld * 8, X.data(), ld * 8, nev * 8, n,
                                    cudaMemcpyDeviceToDevice, s));
    csr_spmm<double>(A, V.data(), ld, AV.data(), ld, nullptr, 0, nev, 1.0, 0.0, 0.0, s);
    st.spmm_launches += 1;
    FE_CHECK_CUDA(cudaMemset2DAsync(Pm, cap * 8, 0, cap * 8, cap, s));
    gram_block<double>(sm, V.data(), ld, AV.data(), ld, n, nev, nev, Pm, s);
    int64_t cols = nev;
    extract(cols, ritz);
    for (int64_t blk = 1; blk < opt.maxblks; ++blk) {
      std::vector<int32_t> active;
      for (int64_t j = 0; j < nev; ++j)
        if (ritz.rel[j] > locktol) active.push_back(static_cast<int32_t>(j));
      const int64_t cc = static_cast<int64_t>(active.size());
      if (cc == 0 || cols + cc > cap) break;
      DeviceBuffer act(cc * sizeof(int32_t));
      ctx.to_device(act.as<int32_t>(), active.data(), cc);
      gather_columns<double>(R.data(), ld, act.as<int32_t>(), cc, Cb.data(), ld, n, s);
      block_gs(ctx, sm, V.data(), ld, cols, Cb.data(), Cb.data(), n, cc);
      cholqr2_inplace(ctx, sm, Cb.data(), T1.data(), ld, n, cc,
                      "DavidsonSolver: correction-block");
      csr_spmm<double>(A, Cb.data(), ld, ACb.data(), ld, nullptr, 0, cc, 1.0, 0.0, 0.0, s);
      st.spmm_launches += 1;
      // projected[:cols, cols:cols+cc] = V^T A C, mirrored; diagonal block C^T A C.
      gram_block<double>(sm, V.data(), ld, ACb.data(), ld, n, cols, cc, Pm + cols * cap, s);
      gram_block<double>(sm, Cb.data(), ld, ACb.data(), ld, n, cc, cc, Pm + cols * cap + cols, s);
      mirror_block(Pm, cap, cols, cols, cc, s);
      FE_CHECK_CUDA(cudaMemcpy2DAsync(V.col(cols), ld * 8, Cb.data(), ld * 8, cc * 8, n,
                                      cudaMemcpyDeviceToDevice, s));
      FE_CHECK_CUDA(cudaMemcpy2DAsync(AV.col(cols), ld * 8, ACb.data(), ld * 8, cc * 8, n,
                                      cudaMemcpyDeviceToDevice, s));
      cols += cc;
      extract(cols, ritz);
    }
    it_done = iter + 1;
    double worst = 0;
    for (double v : ritz.rel) worst = std::max(worst, v);
    if (opt.verbosity >= 2)
      std::fprintf(stderr, "[fe] davidson iter %lld cols %lld worst %.3e\n",
                   static_cast<long long>(iter + 1), static_cast<long long>(cols), worst);
    if (!ritz.rel.empty() && worst < tol) break;
  }
  for (int64_t j = 0; j < nev; ++j) eigenvalues[j] = ritz.values[j];
  finish_results(ctx, sm, A, nullptr, X.data(), ld, n, nev, eigenvalues, residuals, eigenvectors);
  st.iterations = static_cast<double>(it_done);
  st.fp64_iterations = static_cast<double>(it_done);
}

void check_pair(const Csr& A, const Csr& B) {
  FE_REQUIRE(B.rows == A.rows && B.cols == A.cols,
             "generalized problem: B must have the same shape as A.");
  FE_REQUIRE(B.device == A.device, "generalized problem: A and B live on different devices.");
}

// ===========================================================================
// Extension: generalized K u = l M u and Jacobi-preconditioned LOBPCG / block
// Davidson (the reference's solvers are standard-only and unpreconditioned,
// src/LOBPCGSolver.cpp:25-174, src/DavidsonSolver.cpp:27-264). Same loops with
// every inner product in the B metric (the weighted Gram of the reference's
// weighted Cholesky QR, src/core/Orthogonalization.cpp:407-440), corrections
// W = T R with T = diag(|K_ii|)^-1, and the relative residual of
// evaluate_ritz_pairs with B (src/core/RitzExtraction.cpp:50-56). B absent means
// M = I (B-blocks are then copies).
// ===========================================================================
template <typename T>
struct GenBlockOpsT {
  Context& ctx;
  SmallState& sm;
  ProjectedEig& eig;
  const Csr& A;
  const Csr* B;
  double sign;
  int64_t n, ld;
  Stats& st;
  DeviceBuffer idx_dev;
  // Singular values of an orthonormalization below this fraction of the largest
  // are dropped as noise: about sqrt(unit roundoff) of the block's precision.
  static constexpr double kRankFloor = sizeof(T) == 4 ? 1e-3 : 1e-7;

  void bapply(const T* X, T* BX, int64_t cols) {
    if (cols <= 0) return;
    if (B) {
      csr_spmm<T>(*B, X, ld, BX, ld, nullptr, 0, cols, 1.0, 0.0, 0.0, ctx.stream);
      st.spmm_launches += 1;
    } else {
      FE_CHECK_CUDA(cudaMemcpy2DAsync(BX, ld * sizeof(T), X, ld * sizeof(T), cols * sizeof(T), n,
                                      cudaMemcpyDeviceToDevice, ctx.stream));
    }
  }
  void happly(const T* X, T* AX, int64_t cols) {
    if (cols <= 0) return;
    csr_spmm<T>(A, X, ld, AX, ld, nullptr, 0, cols, sign, 0.0, 0.0, ctx.stream);
    st.spmm_launches += 1;
  }
  void copy(T* dst, const T* src, int64_t cols) {
    if (cols <= 0 || dst == src) return;
    FE_CHECK_CUDA(cudaMemcpy2DAsync(dst, ld * sizeof(T), src, ld * sizeof(T), cols * sizeof(T), n,
                                    cudaMemcpyDeviceToDevice, ctx.stream));
  }

  // B-orthonormal basis of the part of src (cols columns) outside span(V[:, :k]),
  // V B-orthonormal with BV = B V: two passes of B-norms -> two-pass block
  // Gram-Schmidt in the B metric -> B-Gram eigen-decomposition -> keep singular
  // values above max(rank_tol * largest B-norm, 1e-7 * largest) -> rotate by
  // U S^-1 (orthonormalize_block, src/core/Orthogonalization.cpp:717-775, in the B
  // metric). Writes out/Bout[:, :rank] (may alias src; tmp/tmpB are scratch).
  int64_t ortho(const T* V, const T* BV, int64_t k, const T* src, int64_t cols, T* out, T* Bout,
                T* tmp, T* tmpB, double rank_tol = 1e-12) {
    cudaStream_t s = ctx.stream;
    if (k >= n || cols <= 0) return 0;
    const T* cur = src;
    int64_t rank = 0;
    std::vector<double> norms, w, inv;
    for (int pass = 0; pass < 2; ++pass) {
      bapply(cur, tmpB, cols);
      residual_norms<T>(nullptr, cur, tmpB, ld, n, cols, nullptr, nullptr, 0, nullptr,
                             sm.xnorm.as<double>(), nullptr, sm.rws.get(), sm.rws.bytes(), s, 2);
      norms.resize(cols);
      ctx.to_host(norms.data(), sm.xnorm.as<double>(), cols);
      ctx.sync();
      double scale = 0.0;
      for (double v : norms) {
        if (!std::isfinite(v))
          throw Error(FE_ERR_NONFINITE, "orthonormalize_block: non-finite column norms.");
        scale = std::max(scale, v);
      }
      if (scale == 0.0) return 0;
      copy(tmp, cur, cols);
      double* G = sm.G.as<double>();
      if (k > 0) {
        for (int g = 0; g < 2; ++g) {
          gram_block<T>(sm, V, ld, tmpB, ld, n, k, cols, G, s);
          rotate_block<T>(sm, V, ld, G, tmp, ld, n, k, cols, -1.0, 1.0, s);
          rotate_block<T>(sm, BV, ld, G, tmpB, ld, n, k, cols, -1.0, 1.0, s);
        }
      }
      gram_block<T>(sm, tmp, ld, tmpB, ld, n, cols, cols, G, s);
      symmetrize(G, cols, sm.cap, s);
      eig.run(G, cols, sm.cap, sm.W.as<double>());
      w.resize(cols);
      ctx.to_host(w.data(), sm.W.as<double>(), cols);
      ctx.sync();
      const double smax = std::sqrt(std::max(w[cols - 1], 0.0));
      const int64_t capacity = std::min<int64_t>(cols, n - k);
      const double cut = std::max(rank_tol * scale, kRankFloor * smax);
      std::vector<int32_t> sel;
      inv.clear();
      for (int64_t i = cols - 1; i >= 0 && static_cast<int64_t>(sel.size()) < capacity; --i) {
        const double sv = std::sqrt(std::max(w[i], 0.0));
        if (!(sv > cut)) break;
        sel.push_back(static_cast<int32_t>(i));
        inv.push_back(1.0 / sv);
      }
      rank = static_cast<int64_t>(sel.size());
      if (rank == 0) return 0;
      const size_t dbl_off = ((rank * sizeof(int32_t) + 7) / 8) * 8;
      idx_dev.resize(dbl_off + rank * sizeof(double));
      int32_t* di = idx_dev.as<int32_t>();
      double* ds = reinterpret_cast<double*>(idx_dev.as<uint8_t>() + dbl_off);
      ctx.to_device(di, sel.data(), rank);
      ctx.to_device(ds, inv.data(), rank);
      small_gather_scale(G, sm.cap, cols, di, ds, rank, sm.Rinv.as<double>(), sm.cap, s);
      rotate_block<T>(sm, tmp, ld, sm.Rinv.as<double>(), out, ld, n, cols, rank, 1.0, 0.0, s);
      rotate_block<T>(sm, tmpB, ld, sm.Rinv.as<double>(), Bout, ld, n, cols, rank, 1.0, 0.0, s);
      cur = out;
      cols = rank;
      ctx.sync();
    }
    return rank;
  }

  // Weighted Cholesky QR with a fresh BX: X <- X R^-1, BX <- B X R^-1 (through tmp/tmpB).
  void bcholqr(T* X, T* BX, int64_t b, T* tmp, T* tmpB, const char* what) {
    cudaStream_t s = ctx.stream;
    bapply(X, BX, b);
    double* G = sm.G.as<double>();
    gram_block<T>(sm, X, ld, BX, ld, n, b, b, G, s);
    symmetrize(G, b, sm.cap, s);
    FE_CHECK_CUDA(cudaMemsetAsync(sm.info.get(), 0, sizeof(int32_t), s));
    chol_inverse(G, b, sm.cap, sm.Rinv.as<double>(), sm.cap, sm.info.as<int32_t>(), s);
    int32_t info = 0;
    ctx.to_host(&info, sm.info.as<int32_t>(), 1);
    ctx.sync();
    if (info != 0) throw Error(FE_ERR_NOT_SPD, std::string(what) + ": weighted QR failed.");
    rotate_block<T>(sm, X, ld, sm.Rinv.as<double>(), tmp, ld, n, b, b, 1.0, 0.0, s);
    rotate_block<T>(sm, BX, ld, sm.Rinv.as<double>(), tmpB, ld, n, b, b, 1.0, 0.0, s);
    copy(X, tmp, b);
    copy(BX, tmpB, b);
  }
};
using GenBlockOps = GenBlockOpsT<double>;

// Device blocks of one precision phase of the generalized LOBPCG.
template <typename T>
struct LobpcgBlocks {
  Block<T> X, AX, BX, R, Pd, S, AS, BS, T1, T2, Wsrc;
  void allocate(int64_t n, int64_t cap) {
    for (Block<T>* q : {&X, &AX, &BX, &R, &Pd, &S, &AS, &BS, &T1, &T2, &Wsrc}) q->allocate(n, cap);
  }
};

// One precision phase of the generalized LOBPCG (LOBPCGSolver::solve,
// src/LOBPCGSolver.cpp:25-174, in the B metric with an optional Jacobi
// preconditioner t): B-orthonormalize the start block X[:, :b], Rayleigh-Ritz,
// then iterate until every wanted pair's residual is <= lock_tol (pairs at or
// below it leave the correction block W), maxiter, or, with stop_at_floor (the
// FP32 phase), a worst residual below 1e-3 that has not halved over fifteen
// iterations (far from convergence the worst pair of a LOBPCG block can sit still
// for a while before the block converges; near the FP32 floor it creeps).
template <typename T>
void lobpcg_gen_phase(Context& ctx, SmallState& sm, ProjectedEig& eig, const Csr& A,
                      const Csr* B, const Options& opt, double sign, int64_t b, int64_t cap,
                      const double* t, LobpcgBlocks<T>& L, RitzResult& ritz, int64_t& it_done,
                      double lock_tol, bool stop_at_floor, DeviceBuffer& act, DeviceBuffer& coef,
                      Stats& st) {
  cudaStream_t s = ctx.stream;
  const int64_t n = A.rows, nev = opt.nev, ld = L.X.ld;
  GenBlockOpsT<T> g{ctx, sm, eig, A, B, sign, n, ld, st, DeviceBuffer(64)};
  if (g.ortho(nullptr, nullptr, 0, L.X.data(), b, L.X.data(), L.BX.data(), L.T1.data(),
              L.T2.data()) < b)
    throw Error(FE_ERR_NOT_SPD, "LOBPCGSolver: initial block is rank deficient.");
  g.happly(L.X.data(), L.AX.data(), b);
  g.copy(L.S.data(), L.X.data(), b);
  g.copy(L.AS.data(), L.AX.data(), b);
  g.copy(L.BS.data(), L.BX.data(), b);
  gram_block<T>(sm, L.S.data(), ld, L.AS.data(), ld, n, b, b, sm.G.as<double>(), s);
  ritz_extract<T>(ctx, sm, eig, sm.G.as<double>(), L.S.data(), L.AS.data(), ld, n, b, b, "sr",
                  L.X.data(), L.AX.data(), L.R.data(), coef.as<double>(), g.idx_dev, ritz,
                  L.BS.data(), L.BX.data());
  auto worst_nev = [&] {
    double w = 0;
    for (int64_t j = 0; j < nev; ++j) w = std::max(w, ritz.rel[j]);
    return w;
  };
  std::vector<double> history;
  bool have_p = false;
  while (it_done < opt.maxiter) {
    const double worst = worst_nev();
    if (worst <= lock_tol) break;
    if (stop_at_floor && worst <= 1e-3) {
      history.push_back(worst);
      const size_t h = history.size();
      if (h > 15 && worst > 0.5 * history[h - 16]) break;
    }
    std::vector<int32_t> active;
    for (int64_t j = 0; j < b; ++j)
      if (ritz.rel[j] > lock_tol) active.push_back(static_cast<int32_t>(j));
    const int64_t na = static_cast<int64_t>(active.size());
    ctx.to_device(act.as<int32_t>(), active.data(), na);
    gather_columns<T>(L.R.data(), ld, act.as<int32_t>(), na, L.Wsrc.data(), ld, n, s, t);
    g.bcholqr(L.X.data(), L.BX.data(), b, L.T1.data(), L.T2.data(), "LOBPCGSolver: Ritz-vector");
    g.copy(L.S.data(), L.X.data(), b);
    g.copy(L.BS.data(), L.BX.data(), b);
    int64_t cols = b;
    const int64_t rw = g.ortho(L.S.data(), L.BS.data(), cols, L.Wsrc.data(), na, L.S.col(cols),
                               L.BS.col(cols), L.T1.data(), L.T2.data());
    cols += std::min(rw, cap - cols);
    if (have_p && cols < cap) {
      gather_columns<T>(L.Pd.data(), ld, act.as<int32_t>(), na, L.Wsrc.data(), ld, n, s);
      const int64_t rp = g.ortho(L.S.data(), L.BS.data(), cols, L.Wsrc.data(), na, L.S.col(cols),
                                 L.BS.col(cols), L.T1.data(), L.T2.data());
      cols += std::min(rp, cap - cols);
    }
    g.happly(L.S.data(), L.AS.data(), cols);
    gram_block<T>(sm, L.S.data(), ld, L.AS.data(), ld, n, cols, cols, sm.G.as<double>(), s);
    ritz_extract<T>(ctx, sm, eig, sm.G.as<double>(), L.S.data(), L.AS.data(), ld, n, cols, b, "sr",
                    L.X.data(), L.AX.data(), L.R.data(), coef.as<double>(), g.idx_dev, ritz,
                    L.BS.data(), L.BX.data());
    // P = S C with the X rows of C zeroed.
    FE_CHECK_CUDA(cudaMemset2DAsync(coef.get(), cap * 8, 0, b * 8, b, s));
    rotate_block<T>(sm, L.S.data(), ld, coef.as<double>(), L.Pd.data(), ld, n, cols, b, 1.0, 0.0,
                    s);
    have_p = true;
    ++it_done;
    if (opt.verbosity >= 2)
      std::fprintf(stderr, "[fe] lobpcg-g %s iter %lld cols %lld worst %.3e\n",
                   sizeof(T) == 4 ? "fp32" : "fp64", static_cast<long long>(it_done),
                   static_cast<long long>(cols), worst_nev());
    if (worst_nev() <= lock_tol || cols == b) break;
  }
}

// Generalized / preconditioned / wide-block LOBPCG. precision=mixed runs the
// iteration on FP32 blocks (FP32 SpMMs, split-TF32 Grams and rotations, FP64
// projected problems) until the wanted pairs reach the FP32 floor (mixed_switch)
// or stall there, then restarts from those Ritz vectors on FP64 blocks to tol
// (carrying the FP32 search directions P over measured slower: 78 vs 66 FP64
// iterations on the 80^3 pair).
void lobpcg_gen_solve(const Csr& A, const Csr* B, const Options& opt, double* eigenvalues,
                      double* residuals, double* eigenvectors, Stats& st) {
  const int64_t n = A.rows, nev = opt.nev;
  if (n <= 0 || nev <= 0 || nev > n || opt.maxiter <= 0)
    throw Error(FE_ERR_INVALID, "LOBPCGSolver: require 0 < nev <= n and maxiter > 0.");
  if (opt.which != "sr" && opt.which != "lr")
    throw Error(FE_ERR_INVALID, "LOBPCGSolver: only SR and LR are supported.");
  FE_REQUIRE(opt.precision == "fp64" || opt.precision == "mixed",
             "precision must be fp64 or mixed");
  const int64_t b = std::min<int64_t>(n, std::max<int64_t>(nev, opt.block));
  const double sign = opt.which == "lr" ? -1.0 : 1.0;
  const double tol = opt.tol;
  const int64_t cap = std::min<int64_t>(n, 3 * b);
  const bool mixed = opt.precision == "mixed";
  Context ctx;
  cudaStream_t s = ctx.stream;
  SmallState sm;
  sm.allocate(n, cap, mixed && opt.tensor_cores && tc_gemm_available());
  ProjectedEig eig(ctx, cap);
  DeviceBuffer tdiag, act(static_cast<size_t>(cap) * sizeof(int32_t) + 16),
      coef(static_cast<size_t>(cap) * cap * sizeof(double));
  const double* t = nullptr;
  if (opt.precond == "jacobi") {
    tdiag.resize(n * sizeof(double));
    jacobi_inverse_diagonal(A, tdiag.as<double>(), s);
    t = tdiag.as<double>();
  }
  RitzResult ritz;
  int64_t it_done = 0;
  LobpcgBlocks<double> D;
  if (mixed) {
    LobpcgBlocks<float> F;
    F.allocate(n, cap);
    {
      Block<double> X0;
      X0.allocate(n, b);
      fill_initial_block(ctx, X0.data(), X0.ld, n, b, opt.seed_or_default(), opt.init == "host");
      convert<double, float>(X0.data(), X0.ld, F.X.data(), F.X.ld, n, b, s);
      ctx.sync();
    }
    lobpcg_gen_phase<float>(ctx, sm, eig, A, B, opt, sign, b, cap, t, F, ritz, it_done,
                            std::max(tol, opt.mixed_switch), true, act, coef, st);
    st.fp32_iterations = static_cast<double>(it_done);
    D.allocate(n, cap);
    convert<float, double>(F.X.data(), F.X.ld, D.X.data(), D.X.ld, n, b, s);
    ctx.sync();
  } else {
    D.allocate(n, cap);
    fill_initial_block(ctx, D.X.data(), D.X.ld, n, b, opt.seed_or_default(), opt.init == "host");
  }
  const int64_t it64 = it_done;
  lobpcg_gen_phase<double>(ctx, sm, eig, A, B, opt, sign, b, cap, t, D, ritz, it_done, tol, false,
                           act, coef, st);
  for (int64_t j = 0; j < nev; ++j) eigenvalues[j] = sign * ritz.values[j];
  finish_results(ctx, sm, A, B, D.X.data(), D.X.ld, n, nev, eigenvalues, residuals, eigenvectors);
  st.iterations = static_cast<double>(it_done);
  st.fp64_iterations = static_cast<double>(it_done - it64);
}

template <typename T>
struct DavidsonBlocks {
  Block<T> V, AV, BV, X, AX, BX, R, T1, T2, Wsrc;
  void allocate(int64_t n, int64_t cap) {
    for (Block<T>* q : {&V, &AV, &BV, &X, &AX, &BX, &R, &T1, &T2, &Wsrc}) q->allocate(n, cap);
  }
};

// One precision phase of the generalized block Davidson (DavidsonSolver::solve,
// src/DavidsonSolver.cpp:27-264, in the B metric with an optional Jacobi
// preconditioner t): restart from X[:, :bw], expand the basis by up to maxblks - 1
// blocks of corrections, Rayleigh-Ritz after each. Stops when the wanted pairs are
// below `stop_tol`, at maxiter, or, with stop_at_floor (the FP32 phase), when a
// worst residual below 1e-3 has not halved over eight restarts. Corrections are
// formed for pairs above `active_tol`.
template <typename T>
void davidson_gen_phase(Context& ctx, SmallState& sm, ProjectedEig& eig, const Csr& A,
                        const Csr* B, const Options& opt, int64_t bw, int64_t cap,
                        const double* t, DavidsonBlocks<T>& L, RitzResult& ritz,
                        int64_t& it_done, double stop_tol, double active_tol, bool stop_at_floor,
                        DeviceBuffer& act, DeviceBuffer& coef, DeviceBuffer& proj, Stats& st) {
  cudaStream_t s = ctx.stream;
  const int64_t n = A.rows, nev = opt.nev, ld = L.V.ld;
  const std::string which = opt.which;
  GenBlockOpsT<T> g{ctx, sm, eig, A, B, 1.0, n, ld, st, DeviceBuffer(64)};
  double* Pm = proj.as<double>();
  double* Pw = sm.G.as<double>();
  auto extract = [&](int64_t cols) {
    FE_CHECK_CUDA(cudaMemcpy2DAsync(Pw, cap * 8, Pm, cap * 8, cols * 8, cols,
                                    cudaMemcpyDeviceToDevice, s));
    ritz_extract<T>(ctx, sm, eig, Pw, L.V.data(), L.AV.data(), ld, n, cols, bw, which,
                    L.X.data(), L.AX.data(), L.R.data(), coef.as<double>(), g.idx_dev, ritz,
                    L.BV.data(), L.BX.data());
  };
  if (g.ortho(nullptr, nullptr, 0, L.X.data(), bw, L.X.data(), L.BX.data(), L.T1.data(),
              L.T2.data()) < bw)
    throw Error(FE_ERR_NOT_SPD, "DavidsonSolver: initial block is rank deficient.");
  g.copy(L.V.data(), L.X.data(), bw);
  g.copy(L.BV.data(), L.BX.data(), bw);
  g.happly(L.V.data(), L.AV.data(), bw);
  gram_block<T>(sm, L.V.data(), ld, L.AV.data(), ld, n, bw, bw, Pm, s);
  extract(bw);
  std::vector<double> history;
  while (it_done < opt.maxiter) {
    g.bcholqr(L.X.data(), L.BX.data(), bw, L.T1.data(), L.T2.data(), "DavidsonSolver: restart");
    g.copy(L.V.data(), L.X.data(), bw);
    g.copy(L.BV.data(), L.BX.data(), bw);
    g.happly(L.V.data(), L.AV.data(), bw);
    FE_CHECK_CUDA(cudaMemset2DAsync(Pm, cap * 8, 0, cap * 8, cap, s));
    gram_block<T>(sm, L.V.data(), ld, L.AV.data(), ld, n, bw, bw, Pm, s);
    int64_t cols = bw;
    extract(cols);
    for (int64_t blk = 1; blk < opt.maxblks; ++blk) {
      std::vector<int32_t> active;
      for (int64_t j = 0; j < bw; ++j)
        if (ritz.rel[j] > active_tol) active.push_back(static_cast<int32_t>(j));
      const int64_t cc = static_cast<int64_t>(active.size());
      if (cc == 0 || cols + cc > cap) break;
      ctx.to_device(act.as<int32_t>(), active.data(), cc);
      gather_columns<T>(L.R.data(), ld, act.as<int32_t>(), cc, L.Wsrc.data(), ld, n, s, t);
      const int64_t r = g.ortho(L.V.data(), L.BV.data(), cols, L.Wsrc.data(), cc, L.V.col(cols),
                                L.BV.col(cols), L.T1.data(), L.T2.data());
      if (r == 0) break;
      g.happly(L.V.col(cols), L.AV.col(cols), r);
      // projected[:cols, cols:cols+r] = V^T A W, mirrored; diagonal block W^T A W.
      gram_block<T>(sm, L.V.data(), ld, L.AV.col(cols), ld, n, cols, r, Pm + cols * cap, s);
      gram_block<T>(sm, L.V.col(cols), ld, L.AV.col(cols), ld, n, r, r, Pm + cols * cap + cols,
                    s);
      mirror_block(Pm, cap, cols, cols, r, s);
      cols += r;
      extract(cols);
    }
    ++it_done;
    double worst = 0;
    for (int64_t j = 0; j < nev; ++j) worst = std::max(worst, ritz.rel[j]);
    if (opt.verbosity >= 2)
      std::fprintf(stderr, "[fe] davidson-g %s iter %lld cols %lld worst %.3e\n",
                   sizeof(T) == 4 ? "fp32" : "fp64", static_cast<long long>(it_done),
                   static_cast<long long>(cols), worst);
    if (!ritz.rel.empty() && worst < stop_tol) break;
    if (stop_at_floor && worst <= 1e-3) {
      history.push_back(worst);
      const size_t h = history.size();
      if (h > 8 && worst > 0.5 * history[h - 9]) break;
    }
  }
}

// Generalized / preconditioned / wide-block Davidson. precision=mixed runs the
// restarts on FP32 blocks (FP32 SpMMs, split-TF32 Grams and rotations, FP64
// projected problems) until the wanted pairs reach the FP32 floor (mixed_switch)
// or stall there, then restarts from those Ritz vectors on FP64 blocks to tol.
void davidson_gen_solve(const Csr& A, const Csr* B, const Options& opt, double* eigenvalues,
                        double* residuals, double* eigenvectors, Stats& st) {
  const int64_t n = A.rows, nev = opt.nev;
  if (n <= 0) throw Error(FE_ERR_INVALID, "DavidsonSolver: n must be > 0.");
  if (nev <= 0 || nev > n) throw Error(FE_ERR_INVALID, "DavidsonSolver: nev must be in [1,n].");
  if (opt.maxiter <= 0) throw Error(FE_ERR_INVALID, "DavidsonSolver: maxiter must be > 0.");
  if (opt.maxblks < 1) throw Error(FE_ERR_INVALID, "DavidsonSolver: maxblks must be at least 1.");
  const std::string which = opt.which;
  if (which != "sr" && which != "lr" && which != "sm" && which != "lm" && which != "be")
    throw Error(FE_ERR_INVALID, "DavidsonSolver: invalid which option (use SR/LR/SM/LM/BE).");
  FE_REQUIRE(opt.precision == "fp64" || opt.precision == "mixed",
             "precision must be fp64 or mixed");
  const double tol = opt.tol;
  const bool mixed = opt.precision == "mixed";
  // Block of b >= nev Ritz vectors; convergence is judged on the first nev.
  const int64_t bw = std::min<int64_t>(n, std::max<int64_t>(nev, opt.block));
  const int64_t cap = std::min<int64_t>(n, opt.maxblks * bw);
  Context ctx;
  cudaStream_t s = ctx.stream;
  SmallState sm;
  sm.allocate(n, cap, mixed && opt.tensor_cores && tc_gemm_available());
  ProjectedEig eig(ctx, cap);
  DeviceBuffer tdiag, act(static_cast<size_t>(cap) * sizeof(int32_t) + 16),
      coef(static_cast<size_t>(cap) * cap * sizeof(double)),
      proj(static_cast<size_t>(cap) * cap * sizeof(double));
  const double* t = nullptr;
  if (opt.precond == "jacobi") {
    tdiag.resize(n * sizeof(double));
    jacobi_inverse_diagonal(A, tdiag.as<double>(), s);
    t = tdiag.as<double>();
  }
  RitzResult ritz;
  int64_t it_done = 0;
  DavidsonBlocks<double> D;
  if (mixed) {
    DavidsonBlocks<float> F;
    F.allocate(n, cap);
    {
      Block<double> X0;
      X0.allocate(n, bw);
      fill_initial_block(ctx, X0.data(), X0.ld, n, bw, opt.seed_or_default(), opt.init == "host");
      convert<double, float>(X0.data(), X0.ld, F.X.data(), F.X.ld, n, bw, s);
      ctx.sync();
    }
    const double floor32 = std::max(tol, opt.mixed_switch);
    davidson_gen_phase<float>(ctx, sm, eig, A, B, opt, bw, cap, t, F, ritz, it_done, floor32,
                              floor32, true, act, coef, proj, st);
    st.fp32_iterations = static_cast<double>(it_done);
    D.allocate(n, cap);
    convert<float, double>(F.X.data(), F.X.ld, D.X.data(), D.X.ld, n, bw, s);
    ctx.sync();
  } else {
    D.allocate(n, cap);
    fill_initial_block(ctx, D.X.data(), D.X.ld, n, bw, opt.seed_or_default(), opt.init == "host");
  }
  const int64_t it64 = it_done;
  davidson_gen_phase<double>(ctx, sm, eig, A, B, opt, bw, cap, t, D, ritz, it_done, tol,
                             std::min(1.0e-5, tol), false, act, coef, proj, st);
  for (int64_t j = 0; j < nev; ++j) eigenvalues[j] = ritz.values[j];
  finish_results(ctx, sm, A, B, D.X.data(), D.X.ld, n, nev, eigenvalues, residuals, eigenvectors);
  st.iterations = static_cast<double>(it_done);
  st.fp64_iterations = static_cast<double>(it_done - it64);
}

// Solves B x = b on the device by conjugate gradients with the Jacobi
// preconditioner, to ||r|| <= 1e-14 ||b|| (at most 1000 iterations). Stands in for
// the reference's sparse factorization of B in the generalized Krylov-Schur
// operator B^-1 A (src/gpu/CudaShiftInvertOperator.cpp uses cuDSS): B is the
// symmetric positive definite mass matrix, and its inverse is applied to the
// tolerance of the FP64 path, so the Lanczos recurrence sees B^-1 A to ~1e-14.
struct MassSolver {
  Context& ctx;
  const Csr& B;
  int64_t n;
  DeviceBuffer t, r, z, p, q, out, ws, idx0;
  int64_t iterations = 0;
  MassSolver(Context& c, const Csr& b)
      : ctx(c), B(b), n(b.rows), t(n * 8), r(n * 8), z(n * 8), p(n * 8), q(n * 8), out(8),
        ws(std::max<size_t>(residual_workspace_bytes(b.rows, 1), 64)), idx0(16) {
    jacobi_inverse_diagonal(B, t.as<double>(), ctx.stream);
    const int32_t zero = 0;
    ctx.to_device(idx0.as<int32_t>(), &zero, 1);
  }
  // sqrt(x . y) for x . y >= 0 (the B-norm kernel with y in place of B x).
  double dot_pos(const double* x, const double* y) {
    residual_norms<double>(nullptr, x, y, 1, n, 1, nullptr, nullptr, 0, nullptr, out.as<double>(),
                           nullptr, ws.get(), ws.bytes(), ctx.stream, 2);
    double v = 0;
    ctx.to_host(&v, out.as<double>(), 1);
    ctx.sync();
    return v * v;
  }
  void precondition(const double* src, double* dst) {
    gather_columns<double>(src, 1, idx0.as<int32_t>(), 1, dst, 1, n, ctx.stream, t.as<double>());
  }
  // x = B^-1 b (x and b distinct device vectors).
  void solve(const double* b, double* x) {
    cudaStream_t s = ctx.stream;
    FE_CHECK_CUDA(cudaMemsetAsync(x, 0, n * sizeof(double), s));
    FE_CHECK_CUDA(cudaMemcpyAsync(r.get(), b, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    const double bnorm2 = dot_pos(b, b);
    if (bnorm2 == 0.0) return;
    precondition(r.as<double>(), z.as<double>());
    FE_CHECK_CUDA(cudaMemcpyAsync(p.get(), z.get(), n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    double rz = dot_pos(r.as<double>(), z.as<double>());
    for (int it = 0; it < 1000; ++it) {
      csr_spmm<double>(B, p.as<double>(), 1, q.as<double>(), 1, nullptr, 0, 1, 1.0, 0.0, 0.0, s);
      const double pq = dot_pos(p.as<double>(), q.as<double>());
      if (!(pq > 0.0) || !std::isfinite(pq))
        throw Error(FE_ERR_NONFINITE, "B must be positive definite (invalid B-norm).");
      const double alpha = rz / pq;
      vec_axpby(n, alpha, p.as<double>(), 1, 1.0, x, 1, s);
      vec_axpby(n, -alpha, q.as<double>(), 1, 1.0, r.as<double>(), 1, s);
      ++iterations;
      if (dot_pos(r.as<double>(), r.as<double>()) <= 1e-28 * bnorm2) return;
      precondition(r.as<double>(), z.as<double>());
      const double rz_new = dot_pos(r.as<double>(), z.as<double>());
      vec_axpby(n, 1.0, z.as<double>(), 1, rz_new / rz, p.as<double>(), 1, s);
      rz = rz_new;
    }
    throw Error(FE_ERR_NONFINITE, "KrylovSchurSolver: mass-matrix solve did not converge.");
  }
};

// KrylovSchurSolver::solve (src/KrylovSchurSolver.cpp:28-160): scalar Lanczos with
// two-pass classical reorthogonalization (KrylovSubspace, src/core/KrylovSubspace.cpp:
// 125-259) on the device, the m x m projected eigenproblem on the host, Krylov-Schur
// restarts that keep the wanted Ritz vectors and a dense coupling row
// (CpuLanczosWorkspace::prepare_krylov_schur_restart, src/core/LanczosWorkspace.cpp:94-107),
// and final Ritz pairs evaluated on the device (evaluate_ritz_pairs,
// src/core/RitzExtraction.cpp:34-63). With B the recurrence runs in the B inner
// product on the operator B^-1 A (B-norms of KrylovSubspace::residual_norm,
// src/core/KrylovSubspace.cpp:162-178; Gram-Schmidt weighted by BV), converged pairs are
// verified by their true residual ||A y - l B y|| / ((1+|l|) ||B y||) and the status is 1
// when they are not (src/KrylovSchurSolver.cpp:136-140).
// Scalar Lanczos recurrence of KrylovSubspace::build_one (src/core/KrylovSubspace.cpp:
// 125-259) on the device: basis V (n x cap, and BV = B V in the B metric), residual f,
// two-pass classical Gram-Schmidt, a fresh seeded random vector on breakdown
// (restart_residual, :251-259), and the projected tridiagonal T (column-major, on the
// host) that the Krylov-Schur and plain Lanczos drivers diagonalize. In the generalized
// case the operator is B^-1 A with B^-1 applied by conjugate gradients (MassSolver).
struct ScalarLanczos {
  Context& ctx;
  const Csr& A;
  const Csr* B;
  int64_t n, cap;
  unsigned seed;
  bool host_init;
  Stats& st;
  cudaStream_t s;
  Block<double> V, BV;
  int64_t ld = 0;
  DeviceBuffer f, w, h, hs, nrm, bf, aw, gws, rws;
  std::unique_ptr<MassSolver> mass;
  std::vector<double> T;
  double beta_next = 0.0;
  int64_t restart_row = -1;

  ScalarLanczos(Context& c, const Csr& A_, const Csr* B_, int64_t cap_, unsigned seed_,
                bool host_init_, Stats& st_)
      : ctx(c), A(A_), B(B_), n(A_.rows), cap(cap_), seed(seed_), host_init(host_init_), st(st_),
        s(c.stream) {
    V.allocate(n, cap);
    if (B) BV.allocate(n, cap);
    ld = V.ld;
    f.resize(n * sizeof(double));
    w.resize(n * sizeof(double));
    h.resize(cap * sizeof(double));
    hs.resize(cap * sizeof(double));
    nrm.resize(sizeof(double));
    if (B) {
      bf.resize(n * sizeof(double));
      aw.resize(n * sizeof(double));
      mass.reset(new MassSolver(ctx, *B));
    }
    gws.resize(std::max<size_t>(gram_workspace_bytes(n, cap, 1), 64));
    rws.resize(std::max<size_t>(residual_workspace_bytes(n, cap), 64));
    T.assign(static_cast<size_t>(cap) * cap, 0.0);
    random_into(f.as<double>(), seed);
  }
  double& t(int64_t r, int64_t c) { return T[static_cast<size_t>(c) * cap + r]; }
  void random_into(double* dst, unsigned sd) {
    if (host_init) {
      std::mt19937 rng(sd);
      std::uniform_real_distribution<double> dist(-1.0, 1.0);
      std::vector<double> v(n);
      for (auto& x : v) x = dist(rng);
      ctx.to_device(dst, v.data(), n);
    } else {
      fill_uniform<double>(dst, 1, n, 1, sd, s);
    }
  }
  // ||x|| (standard) or the B-norm sqrt(x . Bx) with Bx kept in bf (generalized).
  double norm(const double* x) {
    if (B) {
      csr_spmm<double>(*B, x, 1, bf.as<double>(), 1, nullptr, 0, 1, 1.0, 0.0, 0.0, s);
      st.spmm_launches += 1;
      residual_norms<double>(nullptr, x, bf.as<double>(), 1, n, 1, nullptr, nullptr, 0, nullptr,
                             nrm.as<double>(), nullptr, rws.get(), rws.bytes(), s, 2);
    } else {
      residual_norms<double>(nullptr, x, nullptr, 1, n, 1, nullptr, nullptr, 0, nullptr,
                             nrm.as<double>(), nullptr, rws.get(), rws.bytes(), s, 0);
    }
    double r = 0;
    ctx.to_host(&r, nrm.as<double>(), 1);
    ctx.sync();
    return r;
  }
  // f = src - V_k (W_k^T src), twice (W = BV with B, else V); returns the last coefficient.
  double orthogonalize(int64_t k, const double* src) {
    const double* W = B ? BV.data() : V.data();
    vec_axpby(n, 1.0, src, 1, 0.0, f.as<double>(), 1, s);
    if (k == 0) return 0.0;
    gram<double>(W, ld, f.as<double>(), 1, n, k, 1, h.as<double>(), k, gws.get(), gws.bytes(), s);
    rotate<double>(V.data(), ld, h.as<double>(), k, f.as<double>(), 1, n, k, 1, -1.0, 1.0, s);
    gram<double>(W, ld, f.as<double>(), 1, n, k, 1, hs.as<double>(), k, gws.get(), gws.bytes(),
                 s);
    rotate<double>(V.data(), ld, hs.as<double>(), k, f.as<double>(), 1, n, k, 1, -1.0, 1.0, s);
    double a = 0, b = 0;
    ctx.to_host(&a, h.as<double>() + k - 1, 1);
    ctx.to_host(&b, hs.as<double>() + k - 1, 1);
    ctx.sync();
    return a + b;
  }
  // Basis columns [begin, end): normalize the residual into V[:, col], apply the
  // operator, orthogonalize, record alpha and beta in T.
  void expand(int64_t begin, int64_t end) {
    for (int64_t col = begin; col < end; ++col) {
      bool restarted = false;
      double beta = norm(f.as<double>());
      if (!std::isfinite(beta))
        throw Error(FE_ERR_NONFINITE, "core::KrylovSubspace: non-finite residual norm encountered.");
      if (!(beta > std::numeric_limits<double>::epsilon())) {
        DeviceBuffer cand(n * sizeof(double));
        random_into(cand.as<double>(), seed + static_cast<unsigned>(col + 1));
        orthogonalize(col, cand.as<double>());
        restarted = true;
        beta = norm(f.as<double>());
        if (!(beta > std::numeric_limits<double>::epsilon()))
          throw Error(FE_ERR_NONFINITE,
                      "core::KrylovSubspace: breakdown, unable to generate new basis vector.");
      }
      vec_axpby(n, 1.0 / beta, f.as<double>(), 1, 0.0, V.col(col), ld, s);
      if (B) vec_axpby(n, 1.0 / beta, bf.as<double>(), 1, 0.0, BV.col(col), ld, s);
      if (B) {
        csr_spmm<double>(A, V.col(col), ld, aw.as<double>(), 1, nullptr, 0, 1, 1.0, 0.0, 0.0, s);
        mass->solve(aw.as<double>(), w.as<double>());
      } else {
        csr_spmm<double>(A, V.col(col), ld, w.as<double>(), 1, nullptr, 0, 1, 1.0, 0.0, 0.0, s);
      }
      st.spmm_launches += 1;
      const double alpha = orthogonalize(col + 1, w.as<double>());
      beta_next = norm(f.as<double>());
      if (!std::isfinite(beta_next))
        throw Error(FE_ERR_NONFINITE, "core::KrylovSubspace: non-finite next residual norm encountered.");
      const double rec_beta = restarted ? 0.0 : beta;
      if (col != 0 && col != restart_row) {
        t(col, col - 1) = rec_beta;
        t(col - 1, col) = rec_beta;
      }
      t(col, col) = alpha;
      if (col == restart_row) restart_row = -1;
    }
  }
};

// LanczosSolver::solve (src/LanczosSolver.cpp:29-163): one scalar Lanczos chain of up to
// maxiter basis vectors with full two-pass reorthogonalization and no restart. From nev
// vectors on, every check_every-th step (print_every, else 5) and at maxiter, the
// projected tridiagonal is diagonalized and the chain stops when the nev wanted Ritz
// pairs' estimates |beta_m z_{m-1,j}| / (1 + |theta_j|) are all below tol (in the B
// metric the formed pairs must also pass their true residual check, and a chain that
// broke down keeps going to recover multiplicity). The returned pairs are formed from
// the basis on the device and their residuals recomputed (evaluate_ritz_pairs).
void lanczos_solve(const Csr& A, const Csr* B, const Options& opt, double* eigenvalues,
                   double* residuals, double* eigenvectors, Stats& st) {
  const int64_t n = A.rows, nev = opt.nev, maxiter = opt.maxiter;
  if (maxiter <= 0) throw Error(FE_ERR_INVALID, "LanczosSolver: maxiter must be > 0.");
  if (nev <= 0) throw Error(FE_ERR_INVALID, "LanczosSolver: nev must be > 0.");
  if (maxiter < nev) throw Error(FE_ERR_INVALID, "LanczosSolver: maxiter must be >= nev.");
  if (maxiter > n) throw Error(FE_ERR_INVALID, "LanczosSolver: maxiter must be <= n.");
  const std::string which = opt.which;
  if (which == "sai")
    throw Error(FE_ERR_UNSUPPORTED,
                "LanczosSolver: SAI needs a shift-invert factorization (out of scope here).");
  if (which != "sr" && which != "lr" && which != "sm" && which != "lm" && which != "be")
    throw Error(FE_ERR_INVALID, "LanczosSolver: invalid which option (use SR/LR/SM/LM/BE/SAI).");
  const double tol = opt.tol;
  const int64_t check_every = opt.print_every > 0 ? opt.print_every : 5;
  Context ctx;
  cudaStream_t s = ctx.stream;
  SmallState sm;
  sm.allocate(n, nev, false);
  ScalarLanczos lz(ctx, A, B, maxiter, opt.seed_or_default(), opt.init == "host", st);
  Block<double> Y;
  Y.allocate(n, nev);
  DeviceBuffer C(static_cast<size_t>(maxiter) * nev * sizeof(double));
  // Ritz values (wanted order), their estimates, and the selected eigenvectors of T_m:
  // the projected matrix is tridiagonal, so only the eigenvalues the selection can
  // need are found (bisection) and only the wanted vectors (inverse iteration).
  std::vector<double> lam_s, rel_s, Cs;
  auto snapshot = [&](int64_t m) {
    std::vector<double> dd(m), ee(m > 1 ? m - 1 : 0);
    for (int64_t i = 0; i < m; ++i) dd[i] = lz.t(i, i);
    for (int64_t i = 0; i + 1 < m; ++i) ee[i] = lz.t(i + 1, i);
    TridiagEig tr(dd, ee, static_cast<int>(m));
    const std::vector<int> cand =
        tridiag_candidates(tr, static_cast<int>(nev), which.c_str());
    std::vector<double> cw(cand.size());
    for (size_t c = 0; c < cand.size(); ++c) cw[c] = tr.eigenvalue(cand[c]);
    const std::vector<int32_t> order = select_indices(cw, which);
    const int64_t k = std::min(nev, m);
    lam_s.assign(k, 0.0);
    rel_s.assign(k, 0.0);
    Cs.assign(static_cast<size_t>(m) * k, 0.0);
    std::vector<std::vector<double>> vecs(k);
    for (int64_t j = 0; j < k; ++j) {
      const double theta = cw[order[j]];
      std::vector<const std::vector<double>*> cluster;
      for (int64_t i = 0; i < j; ++i)
        if (std::fabs(lam_s[i] - theta) <= 1e-3 * tr.tnorm) cluster.push_back(&vecs[i]);
      vecs[j] = tr.vector(theta, static_cast<unsigned>(j), cluster);
      lam_s[j] = theta;
      rel_s[j] = std::fabs(lz.beta_next * vecs[j][m - 1]) / (1.0 + std::fabs(theta));
      std::copy(vecs[j].begin(), vecs[j].end(), Cs.begin() + static_cast<size_t>(j) * m);
    }
  };
  // evaluate_ritz_pairs: Y = V[:, :m] Csel, residuals of the formed pairs
  std::vector<double> vals(nev), res(nev), vecs;
  auto form = [&](int64_t m) {
    ctx.to_device(C.as<double>(), Cs.data(), Cs.size());
    rotate<double>(lz.V.data(), lz.ld, C.as<double>(), m, Y.data(), Y.ld, n, m, nev, 1.0, 0.0,
                   s);
    std::copy(lam_s.begin(), lam_s.end(), vals.begin());
    if (eigenvectors) vecs.resize(static_cast<size_t>(n) * nev);
    finish_results(ctx, sm, A, B, Y.data(), Y.ld, n, nev, vals.data(), res.data(),
                   eigenvectors ? vecs.data() : nullptr);
    bool ok = true;
    for (double r : res) ok = ok && r <= tol;
    return ok;
  };
  bool breakdown = false, converged = false, formed = false, verified = false;
  int64_t it_stop = maxiter;
  for (int64_t it = 0; it < maxiter; ++it) {
    lz.expand(it, it + 1);
    const double alpha = lz.t(it, it);
    const double beta = it > 0 ? lz.t(it, it - 1) : 0.0;
    breakdown = breakdown || lz.beta_next <= 64.0 * std::numeric_limits<double>::epsilon() *
                                                 std::max({1.0, std::fabs(alpha), std::fabs(beta)});
    const int64_t m = it + 1;
    const bool do_check = m >= nev && (m % check_every == 0 || m == maxiter);
    if (!do_check) continue;
    const bool resolve_multiplicity = B && breakdown && m < maxiter;
    snapshot(m);
    double worst = 0.0;
    for (double r : rel_s) worst = std::max(worst, r);
    if (opt.verbosity >= 2)
      std::fprintf(stderr, "[fe] lanczos step %lld worst estimate %.3e\n",
                   static_cast<long long>(m), worst);
    if (!resolve_multiplicity && worst < tol) {
      if (B) {
        verified = form(m);
        formed = true;
        if (!verified) continue;
      }
      converged = true;
      it_stop = m;
      break;
    }
  }
  if (!converged) snapshot(maxiter);
  if (!formed || !converged) verified = form(it_stop);
  for (int64_t j = 0; j < nev; ++j) {
    eigenvalues[j] = vals[j];
    residuals[j] = res[j];
  }
  if (eigenvectors) std::memcpy(eigenvectors, vecs.data(), vecs.size() * sizeof(double));
  st.status = (B && !verified) ? 1 : 0;
  st.iterations = static_cast<double>(it_stop);
  st.fp64_iterations = st.iterations;
}

void krylov_schur_solve(const Csr& A, const Csr* B, const Options& opt, double* eigenvalues,
                        double* residuals, double* eigenvectors, Stats& st) {
  const int64_t n = A.rows, nev = opt.nev;
  if (n <= 0) throw Error(FE_ERR_INVALID, "KrylovSchurSolver: n must be > 0.");
  if (nev <= 0 || nev > n) throw Error(FE_ERR_INVALID, "KrylovSchurSolver: nev must be in [1,n].");
  if (opt.maxiter <= 0) throw Error(FE_ERR_INVALID, "KrylovSchurSolver: maxiter must be > 0.");
  const std::string which = opt.which;
  if (which == "sai")
    throw Error(FE_ERR_UNSUPPORTED,
                "KrylovSchurSolver: SAI needs a shift-invert factorization (out of scope here).");
  if (which != "sr" && which != "lr" && which != "sm" && which != "lm" && which != "be")
    throw Error(FE_ERR_INVALID, "KrylovSchurSolver: invalid which option (use SR/LR/SM/LM/BE/SAI).");
  const double tol = opt.tol;
  const int64_t m = std::min<int64_t>(std::max<int64_t>({2 * nev, 20, opt.maxdim}), n);
  Context ctx;
  cudaStream_t s = ctx.stream;
  SmallState sm;
  sm.allocate(n, m, false);
  ScalarLanczos lz(ctx, A, B, m, opt.seed_or_default(), opt.init == "host", st);
  Block<double>& V = lz.V;
  Block<double>& BV = lz.BV;
  Block<double> Y;
  Y.allocate(n, m);
  const int64_t ld = lz.ld;
  DeviceBuffer C(static_cast<size_t>(m) * m * sizeof(double));
  std::vector<double>& T = lz.T;
  auto t = [&](int64_t r, int64_t c) -> double& { return lz.t(r, c); };
  lz.expand(0, m);
  std::unique_ptr<ProjectedEig> deig;
  DeviceBuffer Td;
  if (m > 96) {  // large projected matrices: the device eigensolver
    deig.reset(new ProjectedEig(ctx, m));
    Td.resize(static_cast<size_t>(m) * m * sizeof(double));
  }
  for (int64_t iter = 1; iter <= opt.maxiter; ++iter) {
    std::vector<double> lam, Z;
    if (deig) {
      ctx.to_device(Td.as<double>(), T.data(), T.size());
      deig->run(Td.as<double>(), m, m, sm.W.as<double>());
      lam.resize(m);
      Z.resize(T.size());
      ctx.to_host(lam.data(), sm.W.as<double>(), m);
      ctx.to_host(Z.data(), Td.as<double>(), Z.size());
      ctx.sync();
    } else {
      host_symmetric_eig(T, static_cast<int>(m), lam, Z);
    }
    const std::vector<int32_t> idx = select_indices(lam, which);
    std::vector<double> lam_s(m), rel_s(m);
    for (int64_t j = 0; j < m; ++j) {
      lam_s[j] = lam[idx[j]];
      rel_s[j] = std::fabs(lz.beta_next * Z[static_cast<size_t>(idx[j]) * m + m - 1]) /
                 (1.0 + std::fabs(lam_s[j]));
    }
    int64_t nconv = 0;
    for (int64_t j = 0; j < nev; ++j) {
      const double mag = std::fabs(lam_s[j]);
      const bool ok = B ? rel_s[j] <= tol : rel_s[j] * (1.0 + mag) < tol * mag;
      if (ok) ++nconv;
    }
    const bool at_limit = (m == n) || (iter == opt.maxiter);
    if (opt.verbosity >= 2)
      std::fprintf(stderr, "[fe] krylov-schur restart %lld nconv %lld\n",
                   static_cast<long long>(iter), static_cast<long long>(nconv));
    if (nconv >= nev || at_limit) {
      // evaluate_ritz_pairs: Y = V Csel, R = A Y - B Y diag(l), rel = ||r|| / ((1+|l|) ||B y||)
      std::vector<double> Cs(static_cast<size_t>(m) * nev);
      for (int64_t j = 0; j < nev; ++j)
        std::memcpy(&Cs[static_cast<size_t>(j) * m], &Z[static_cast<size_t>(idx[j]) * m],
                    m * sizeof(double));
      ctx.to_device(C.as<double>(), Cs.data(), Cs.size());
      rotate<double>(V.data(), ld, C.as<double>(), m, Y.data(), Y.ld, n, m, nev, 1.0, 0.0, s);
      std::vector<double> vals(lam_s.begin(), lam_s.begin() + nev), res(nev);
      std::vector<double> vecs;
      if (eigenvectors) vecs.resize(static_cast<size_t>(n) * nev);
      finish_results(ctx, sm, A, B, Y.data(), Y.ld, n, nev, vals.data(), res.data(),
                     eigenvectors ? vecs.data() : nullptr);
      bool verified = true;
      for (double r : res) verified = verified && r <= tol;
      if (!B || verified || at_limit) {
        for (int64_t j = 0; j < nev; ++j) {
          eigenvalues[j] = vals[j];
          residuals[j] = res[j];
        }
        if (eigenvectors) std::memcpy(eigenvectors, vecs.data(), vecs.size() * sizeof(double));
        st.status = (B && !verified) ? 1 : 0;
        st.iterations = static_cast<double>(iter);
        st.fp64_iterations = static_cast<double>(iter);
        return;
      }
    }
    const int64_t spare = (m - nev) / 2;
    int64_t retained = nev + std::min(nconv, spare);
    if (retained == 1 && m > 3) retained = m / 2;
    // rotate_basis: V[:, :retained] = V * C_all[:, :retained] (and BV alike)
    std::vector<double> Cr(static_cast<size_t>(m) * retained);
    for (int64_t j = 0; j < retained; ++j)
      std::memcpy(&Cr[static_cast<size_t>(j) * m], &Z[static_cast<size_t>(idx[j]) * m],
                  m * sizeof(double));
    ctx.to_device(C.as<double>(), Cr.data(), Cr.size());
    rotate<double>(V.data(), ld, C.as<double>(), m, Y.data(), Y.ld, n, m, retained, 1.0, 0.0, s);
    FE_CHECK_CUDA(cudaMemcpy2DAsync(V.data(), ld * 8, Y.data(), Y.ld * 8, retained * 8, n,
                                    cudaMemcpyDeviceToDevice, s));
    if (B) {
      rotate<double>(BV.data(), ld, C.as<double>(), m, Y.data(), Y.ld, n, m, retained, 1.0, 0.0,
                     s);
      FE_CHECK_CUDA(cudaMemcpy2DAsync(BV.data(), ld * 8, Y.data(), Y.ld * 8, retained * 8, n,
                                      cudaMemcpyDeviceToDevice, s));
    }
    std::fill(T.begin(), T.end(), 0.0);
    for (int64_t j = 0; j < retained; ++j) {
      t(j, j) = lam_s[j];
      const double coupling = lz.beta_next * Z[static_cast<size_t>(idx[j]) * m + m - 1];
      t(retained, j) = coupling;
      t(j, retained) = coupling;
    }
    lz.restart_row = retained;
    lz.expand(retained, m);
  }
  throw Error(FE_ERR_INVALID, "KrylovSchurSolver: unreachable solve termination.");
}

// ===========================================================================
// Block Krylov-Schur: BlockKrylovSchurSolver::solve (src/BlockKrylovSchurSolver.cpp:26-215)
// for standard problems, on the device block kernels: the BlockKrylovSubspace
// expansion (src/core/KrylovSubspace.cpp:261-437: block SpMM, two-pass block
// Gram-Schmidt, complete_block_qr of the residual block), the block-tridiagonal
// projection (src/core/LanczosWorkspace.cpp:42-73), residual estimates from the last
// coupling block (src/core/RitzExtraction.cpp:272-380), and the thick block restart
// (src/core/LanczosWorkspace.cpp:109-135). Large blocks stay on the device; the
// projected matrix and the b x b couplings are small host arrays, as in the reference.
// ===========================================================================
void block_krylov_schur_solve(const Csr& A, const Options& opt, double* eigenvalues,
                              double* residuals, double* eigenvectors, Stats& st) {
  const int64_t n = A.rows, nev = opt.nev, b = opt.blksize;
  const std::string which = opt.which;
  if (n <= 0) throw Error(FE_ERR_INVALID, "BlockKrylovSchurSolver: n must be > 0.");
  if (nev <= 0 || nev > n)
    throw Error(FE_ERR_INVALID, "BlockKrylovSchurSolver: nev must be in [1,n].");
  if (opt.maxiter <= 0) throw Error(FE_ERR_INVALID, "BlockKrylovSchurSolver: maxiter must be > 0.");
  if (which == "sai")
    throw Error(FE_ERR_UNSUPPORTED,
                "BlockKrylovSchurSolver: SAI needs a shift-invert factorization (out of scope here).");
  if (which != "sr" && which != "lr" && which != "sm" && which != "lm" && which != "be")
    throw Error(FE_ERR_INVALID, "BlockKrylovSchurSolver: invalid which option.");
  if (b <= 0 || b > n) throw Error(FE_ERR_INVALID, "BlockKrylovSchurSolver: blksize must be in [1,n].");
  const int64_t requested_dim = opt.maxdim > 0 ? opt.maxdim : std::max<int64_t>(2 * nev, 20);
  const int64_t block_count = requested_dim >= n ? 1 + (n - 1) / b : requested_dim / b;
  const int64_t cycle_dim = std::min(n, block_count * b);
  const int64_t wanted_blocks = 1 + (nev - 1) / b;
  if (cycle_dim < n && block_count <= wanted_blocks)
    throw Error(FE_ERR_INVALID,
                "BlockKrylovSchurSolver: maxdim must accommodate ceil(nev/blksize) retained blocks "
                "plus at least one expansion block (or the full matrix dimension).");
  const int64_t pdim = (block_count + 1) * b;  // projection dimension
  const int64_t retained_blocks = cycle_dim == n ? 0 : std::max(wanted_blocks, block_count / 2);
  const int64_t retained_dim = retained_blocks * b;
  const int64_t snapshot_count = std::max(nev, retained_dim);
  const unsigned seed = opt.seed_or_default();
  const bool host_init = opt.init == "host";
  Context ctx;
  cudaStream_t s = ctx.stream;
  SmallState sm;
  sm.allocate(n, pdim, false);
  Block<double> V, Z, Rb, Qb, Y, one, best;
  V.allocate(n, pdim);
  Z.allocate(n, b);
  Rb.allocate(n, b);
  Qb.allocate(n, b);
  Y.allocate(n, std::max<int64_t>(snapshot_count, b));
  one.allocate(n, 1);
  best.allocate(n, 1);
  const int64_t ld = V.ld;
  DeviceBuffer hdev(static_cast<size_t>(pdim) * b * sizeof(double)),
      h2dev(static_cast<size_t>(pdim) * b * sizeof(double)), nrm(sizeof(double)),
      Cd(static_cast<size_t>(pdim) * pdim * sizeof(double));
  FE_CHECK_CUDA(cudaMemsetAsync(V.data(), 0, static_cast<size_t>(n) * ld * sizeof(double), s));
  auto host_random = [&](double* dst, int64_t ldd, int64_t cols, unsigned sd) {
    // Executor::create_random_multivector / create_random_vector (src/core/Executor.cpp:20-62)
    std::mt19937 rng(sd);
    std::uniform_real_distribution<double> dist(-1.0, 1.0);
    std::vector<double> host(static_cast<size_t>(n) * ldd, 0.0);
    for (int64_t j = 0; j < cols; ++j)
      for (int64_t i = 0; i < n; ++i) host[static_cast<size_t>(i) * ldd + j] = dist(rng);
    ctx.to_device(dst, host.data(), host.size());
    ctx.sync();
  };
  auto vnorm = [&](const double* x, int64_t incx) {
    residual_norms<double>(nullptr, x, nullptr, incx, n, 1, nullptr, nullptr, 0, nullptr,
                           nrm.as<double>(), nullptr, sm.rws.get(), sm.rws.bytes(), s, 0);
    double r = 0;
    ctx.to_host(&r, nrm.as<double>(), 1);
    ctx.sync();
    return r;
  };
  // Two-pass classical Gram-Schmidt of the column x (stride ldx) against W[:, :k].
  auto cgs2 = [&](const double* W, int64_t ldw, int64_t k, double* x, int64_t ldx) {
    if (k == 0) return;
    for (int pass = 0; pass < 2; ++pass) {
      gram<double>(W, ldw, x, ldx, n, k, 1, hdev.as<double>(), k, sm.gws.get(), sm.gws.bytes(), s);
      rotate<double>(W, ldw, hdev.as<double>(), k, x, ldx, n, k, 1, -1.0, 1.0, s);
    }
  };
  // complete_block_qr (src/core/Orthogonalization.cpp:609-715) of src (n x b) against
  // V[:, :active] into Q (n x b); R (b x b, column-major host) gets the coupling.
  auto complete_block_qr = [&](int64_t active, const double* src, int64_t lds, double* Q,
                               int64_t ldq, unsigned sd, double reference_norm,
                               std::vector<double>& R) {
    const int64_t capacity = std::min(b, n - active);
    const double threshold = 64.0 * std::numeric_limits<double>::epsilon() * reference_norm;
    R.assign(static_cast<size_t>(b) * b, 0.0);
    if (capacity == b) {
      double* G = sm.G.as<double>();
      int32_t* info = sm.info.as<int32_t>();
      FE_CHECK_CUDA(cudaMemsetAsync(info, 0, sizeof(int32_t), s));
      gram<double>(src, lds, src, lds, n, b, b, G, pdim, sm.gws.get(), sm.gws.bytes(), s);
      potrf_upper(G, b, pdim, info, s);
      int32_t h = 0;
      std::vector<double> Rh(static_cast<size_t>(pdim) * b);
      ctx.to_host(&h, info, 1);
      ctx.to_host(Rh.data(), G, Rh.size());
      ctx.sync();
      if (h == 0) {
        trinv_upper(G, pdim, sm.Rinv.as<double>(), pdim, b, s);
        rotate<double>(src, lds, sm.Rinv.as<double>(), pdim, Q, ldq, n, b, b, 1.0, 0.0, s,
                       /*upper_tri=*/true);
        std::vector<double> g(static_cast<size_t>(b) * b), c(static_cast<size_t>(std::max<int64_t>(active, 1)) * b);
        gram<double>(Q, ldq, Q, ldq, n, b, b, hdev.as<double>(), b, sm.gws.get(), sm.gws.bytes(), s);
        ctx.to_host(g.data(), hdev.as<double>(), g.size());
        if (active > 0) {
          gram<double>(V.data(), ld, Q, ldq, n, active, b, h2dev.as<double>(), active,
                       sm.gws.get(), sm.gws.bytes(), s);
          ctx.to_host(c.data(), h2dev.as<double>(), static_cast<size_t>(active) * b);
        }
        ctx.sync();
        double mind = std::numeric_limits<double>::infinity(), gerr = 0.0, cerr = 0.0;
        bool finite = true;
        for (int64_t j = 0; j < b; ++j) {
          for (int64_t i = 0; i <= j; ++i) {
            const double r = Rh[static_cast<size_t>(j) * pdim + i];
            finite = finite && std::isfinite(r);
            R[static_cast<size_t>(j) * b + i] = r;
          }
          mind = std::min(mind, std::fabs(R[static_cast<size_t>(j) * b + j]));
          for (int64_t i = 0; i < b; ++i) {
            const double v = g[static_cast<size_t>(j) * b + i] - (i == j ? 1.0 : 0.0);
            finite = finite && std::isfinite(v);
            gerr += v * v;
          }
        }
        for (int64_t e = 0; e < active * b; ++e) {
          finite = finite && std::isfinite(c[e]);
          cerr += c[e] * c[e];
        }
        if (finite && mind > threshold && std::sqrt(gerr) < 1e-10 && std::sqrt(cerr) < 1e-10)
          return false;
      }
    }
    // Rank loss: two-pass projection column by column, filling missing directions.
    bool replenished = false;
    FE_CHECK_CUDA(cudaMemset2DAsync(Q, ldq * sizeof(double), 0, b * sizeof(double), n, s));
    for (int64_t j = 0; j < capacity; ++j) {
      double length = 0.0, original_scale = 0.0;
      bool have = false;
      for (int64_t col = 0; col < b; ++col) {
        FE_CHECK_CUDA(cudaMemcpy2DAsync(one.data(), one.ld * sizeof(double), src + col,
                                        lds * sizeof(double), sizeof(double), n,
                                        cudaMemcpyDeviceToDevice, s));
        original_scale = std::max(original_scale, vnorm(one.data(), one.ld));
        cgs2(V.data(), ld, active, one.data(), one.ld);
        cgs2(Q, ldq, j, one.data(), one.ld);
        const double cn = vnorm(one.data(), one.ld);
        if (cn > length) {
          length = cn;
          have = true;
          FE_CHECK_CUDA(cudaMemcpy2DAsync(best.data(), best.ld * sizeof(double), one.data(),
                                          one.ld * sizeof(double), sizeof(double), n,
                                          cudaMemcpyDeviceToDevice, s));
        }
      }
      const double cutoff = std::max(threshold, 1e-12 * original_scale);
      if (have && length > cutoff) {
        FE_CHECK_CUDA(cudaMemcpy2DAsync(one.data(), one.ld * sizeof(double), best.data(),
                                        best.ld * sizeof(double), sizeof(double), n,
                                        cudaMemcpyDeviceToDevice, s));
        length = vnorm(one.data(), one.ld);
      }
      if (!(length > cutoff)) {
        replenished = true;
        length = 0.0;
        for (unsigned attempt = 0; attempt < 4; ++attempt) {
          host_random(one.data(), one.ld, 1, sd + 17u * static_cast<unsigned>(j + 1) + attempt);
          const double rn = vnorm(one.data(), one.ld);
          cgs2(V.data(), ld, active, one.data(), one.ld);
          cgs2(Q, ldq, j, one.data(), one.ld);
          length = vnorm(one.data(), one.ld);
          if (length > 1e-12 * rn) break;
          length = 0.0;
        }
        if (length == 0.0)
          throw Error(FE_ERR_NONFINITE, "complete_block_qr: unable to complete the basis.");
      }
      vec_axpby(n, 1.0 / length, one.data(), one.ld, 0.0, Q + j, ldq, s);
    }
    gram<double>(Q, ldq, src, lds, n, b, b, hdev.as<double>(), b, sm.gws.get(), sm.gws.bytes(), s);
    ctx.to_host(R.data(), hdev.as<double>(), R.size());
    ctx.sync();
    for (int64_t j = 0; j < b; ++j) {
      double c2 = 0.0;
      for (int64_t i = 0; i < b; ++i) c2 += R[static_cast<size_t>(j) * b + i] * R[static_cast<size_t>(j) * b + i];
      if (std::sqrt(c2) <= threshold)
        for (int64_t i = 0; i < b; ++i) R[static_cast<size_t>(j) * b + i] = 0.0;
    }
    return replenished;
  };

  std::vector<double> T(static_cast<size_t>(pdim) * pdim, 0.0), beta(static_cast<size_t>(b) * b, 0.0);
  auto t = [&](int64_t r, int64_t c) -> double& { return T[static_cast<size_t>(c) * pdim + r]; };
  // initialize_basis_block: the seeded block, completed to an orthonormal block.
  {
    if (host_init) host_random(Z.data(), Z.ld, b, seed);
    else fill_uniform<double>(Z.data(), Z.ld, n, b, seed, s);
    std::vector<double> R0;
    complete_block_qr(0, Z.data(), Z.ld, V.data(), ld, seed, 0.0, R0);
  }
  auto expand = [&](int64_t first_block) {
    for (int64_t blk = first_block; blk < block_count; ++blk) {
      csr_spmm<double>(A, V.col(blk * b), ld, Z.data(), Z.ld, nullptr, 0, b, 1.0, 0.0, 0.0, s);
      st.spmm_launches += 1;
      const int64_t active = std::min(n, (blk + 1) * b);
      // block_gram_schmidt (src/core/Orthogonalization.cpp:482-527): two passes.
      FE_CHECK_CUDA(cudaMemcpy2DAsync(Rb.data(), Rb.ld * sizeof(double), Z.data(),
                                      Z.ld * sizeof(double), b * sizeof(double), n,
                                      cudaMemcpyDeviceToDevice, s));
      std::vector<double> H(static_cast<size_t>(active) * b, 0.0), H2(H.size());
      gram<double>(V.data(), ld, Rb.data(), Rb.ld, n, active, b, hdev.as<double>(), active,
                   sm.gws.get(), sm.gws.bytes(), s);
      rotate<double>(V.data(), ld, hdev.as<double>(), active, Rb.data(), Rb.ld, n, active, b, -1.0,
                     1.0, s);
      gram<double>(V.data(), ld, Rb.data(), Rb.ld, n, active, b, h2dev.as<double>(), active,
                   sm.gws.get(), sm.gws.bytes(), s);
      rotate<double>(V.data(), ld, h2dev.as<double>(), active, Rb.data(), Rb.ld, n, active, b,
                     -1.0, 1.0, s);
      ctx.to_host(H.data(), hdev.as<double>(), H.size());
      ctx.to_host(H2.data(), h2dev.as<double>(), H2.size());
      // ||column norms of Z|| for the rank threshold of the residual QR
      std::vector<double> zn(b);
      residual_norms<double>(nullptr, Z.data(), nullptr, Z.ld, n, b, nullptr, nullptr, 0, nullptr,
                             sm.xnorm.as<double>(), nullptr, sm.rws.get(), sm.rws.bytes(), s, 0);
      ctx.to_host(zn.data(), sm.xnorm.as<double>(), b);
      ctx.sync();
      double scale = 0.0;
      for (double x : zn) scale += x * x;
      scale = std::sqrt(scale);
      const int64_t width = 1 + (active - 1) % b;
      const int64_t row = blk * b, nrow = (blk + 1) * b;
      for (int64_t c = 0; c < b; ++c)
        for (int64_t r = 0; r < b; ++r) t(row + r, row + c) = 0.0;
      for (int64_t c = 0; c < width; ++c)
        for (int64_t r = 0; r < width; ++r) {
          const size_t e = static_cast<size_t>(c) * active + (active - width + r);
          t(row + r, row + c) = H[e] + H2[e];
        }
      std::vector<double> R;
      complete_block_qr(std::min(nrow, n), Rb.data(), Rb.ld, V.col(nrow), ld,
                        seed + static_cast<unsigned>(nrow), scale, R);
      for (int64_t c = 0; c < b; ++c)
        for (int64_t r = 0; r < b; ++r) {
          const double v = R[static_cast<size_t>(c) * b + r];
          t(nrow + r, row + c) = v;
          t(row + c, nrow + r) = v;
        }
      beta = R;
    }
  };
  expand(0);
  std::unique_ptr<ProjectedEig> deig;
  DeviceBuffer Td;
  if (cycle_dim > 96) {
    deig.reset(new ProjectedEig(ctx, cycle_dim));
    Td.resize(static_cast<size_t>(cycle_dim) * cycle_dim * sizeof(double));
  }
  const int64_t m = cycle_dim;
  for (int64_t iter = 1; iter <= opt.maxiter; ++iter) {
    std::vector<double> Tm(static_cast<size_t>(m) * m), lam, Zm;
    for (int64_t c = 0; c < m; ++c)
      for (int64_t r = 0; r < m; ++r) Tm[static_cast<size_t>(c) * m + r] = t(r, c);
    if (deig) {
      ctx.to_device(Td.as<double>(), Tm.data(), Tm.size());
      deig->run(Td.as<double>(), m, m, sm.W.as<double>());
      lam.resize(m);
      Zm.resize(Tm.size());
      ctx.to_host(lam.data(), sm.W.as<double>(), m);
      ctx.to_host(Zm.data(), Td.as<double>(), Zm.size());
      ctx.sync();
    } else {
      host_symmetric_eig(Tm, static_cast<int>(m), lam, Zm);
    }
    const std::vector<int32_t> idx = select_indices(lam, which);
    const int64_t cnt = std::min(snapshot_count, m);
    const int64_t tail = 1 + (m - 1) % b;
    std::vector<double> lam_s(cnt), rel_s(cnt);
    for (int64_t j = 0; j < cnt; ++j) {
      lam_s[j] = lam[idx[j]];
      // || beta * y_last ||, y_last = the eigenvector's last `tail` rows (zero padded)
      double a2 = 0.0;
      for (int64_t r = 0; r < b; ++r) {
        double acc = 0.0;
        for (int64_t c = 0; c < tail; ++c)
          acc += beta[static_cast<size_t>(c) * b + r] *
                 Zm[static_cast<size_t>(idx[j]) * m + (m - tail + c)];
        a2 += acc * acc;
      }
      rel_s[j] = std::sqrt(a2) / (1.0 + std::fabs(lam_s[j]));
    }
    const int64_t k = std::min(nev, cnt);
    double worst = 0.0;
    for (int64_t j = 0; j < k; ++j) worst = std::max(worst, rel_s[j]);
    bool converged = k > 0 && worst < opt.tol;
    const bool at_limit = iter == opt.maxiter || cycle_dim == n;
    if (opt.verbosity >= 2)
      std::fprintf(stderr, "[fe] block krylov-schur restart %lld worst %.3e\n",
                   static_cast<long long>(iter), worst);
    if (converged || at_limit) {
      std::vector<double> Cs(static_cast<size_t>(m) * k);
      for (int64_t j = 0; j < k; ++j)
        std::memcpy(&Cs[static_cast<size_t>(j) * m], &Zm[static_cast<size_t>(idx[j]) * m],
                    m * sizeof(double));
      ctx.to_device(Cd.as<double>(), Cs.data(), Cs.size());
      rotate<double>(V.data(), ld, Cd.as<double>(), m, Y.data(), Y.ld, n, m, k, 1.0, 0.0, s);
      std::vector<double> vals(lam_s.begin(), lam_s.begin() + k), res(k);
      std::vector<double> vecs;
      if (eigenvectors) vecs.resize(static_cast<size_t>(n) * k);
      finish_results(ctx, sm, A, nullptr, Y.data(), Y.ld, n, k, vals.data(), res.data(),
                     eigenvectors ? vecs.data() : nullptr);
      converged = true;
      for (double r : res) converged = converged && r <= opt.tol;
      if (converged || at_limit) {
        for (int64_t j = 0; j < k; ++j) {
          eigenvalues[j] = vals[j];
          residuals[j] = res[j];
        }
        if (eigenvectors) std::memcpy(eigenvectors, vecs.data(), vecs.size() * sizeof(double));
        st.status = converged ? 0 : 1;
        st.iterations = static_cast<double>(iter);
        st.fp64_iterations = static_cast<double>(iter);
        return;
      }
    }
    // Thick block restart: V = [V C_keep, Q_residual], T = [diag(theta), F^T; F, .],
    // F = beta * C_keep(last b rows).
    std::vector<double> Cr(static_cast<size_t>(m) * retained_dim), F(static_cast<size_t>(b) * retained_dim);
    for (int64_t j = 0; j < retained_dim; ++j) {
      std::memcpy(&Cr[static_cast<size_t>(j) * m], &Zm[static_cast<size_t>(idx[j]) * m],
                  m * sizeof(double));
      for (int64_t r = 0; r < b; ++r) {
        double acc = 0.0;
        for (int64_t c = 0; c < b; ++c)
          acc += beta[static_cast<size_t>(c) * b + r] * Cr[static_cast<size_t>(j) * m + (m - b + c)];
        F[static_cast<size_t>(j) * b + r] = acc;
      }
    }
    ctx.to_device(Cd.as<double>(), Cr.data(), Cr.size());
    rotate<double>(V.data(), ld, Cd.as<double>(), m, Y.data(), Y.ld, n, m, retained_dim, 1.0, 0.0,
                   s);
    FE_CHECK_CUDA(cudaMemcpy2DAsync(Qb.data(), Qb.ld * sizeof(double), V.col(block_count * b),
                                    ld * sizeof(double), b * sizeof(double), n,
                                    cudaMemcpyDeviceToDevice, s));
    FE_CHECK_CUDA(cudaMemsetAsync(V.data(), 0, static_cast<size_t>(n) * ld * sizeof(double), s));
    FE_CHECK_CUDA(cudaMemcpy2DAsync(V.data(), ld * sizeof(double), Y.data(), Y.ld * sizeof(double),
                                    retained_dim * sizeof(double), n, cudaMemcpyDeviceToDevice, s));
    FE_CHECK_CUDA(cudaMemcpy2DAsync(V.col(retained_dim), ld * sizeof(double), Qb.data(),
                                    Qb.ld * sizeof(double), b * sizeof(double), n,
                                    cudaMemcpyDeviceToDevice, s));
    std::fill(T.begin(), T.end(), 0.0);
    for (int64_t j = 0; j < retained_dim; ++j) {
      t(j, j) = lam_s[j];
      for (int64_t r = 0; r < b; ++r) {
        t(retained_dim + r, j) = F[static_cast<size_t>(j) * b + r];
        t(j, retained_dim + r) = F[static_cast<size_t>(j) * b + r];
      }
    }
    expand(retained_blocks);
  }
  throw Error(FE_ERR_INVALID, "BlockKrylovSchurSolver: unreachable solve termination.");
}

// ===========================================================================
// Batched Krylov-Schur (extension): many independent standard problems, each
// following KrylovSchurSolver::solve (src/KrylovSchurSolver.cpp:28-160) with the
// Lanczos expansion of KrylovSubspace (src/core/KrylovSubspace.cpp:125-259), run
// in lockstep on the grouped kernels of batch_ks.cu. One Lanczos step of the
// whole batch is a captured CUDA graph; the host only acts once per restart
// round (selection, convergence, restart bookkeeping), exactly as the single
// solver does per problem.
// ===========================================================================
struct BatchStats {
  double seconds = 0, rounds = 0, steps = 0, graph_launches = 0;
};

void batch_krylov_schur(const std::vector<const Csr*>& As, const std::vector<int64_t>& nevs,
                        const Options& opt, double* eigenvalues, double* residuals,
                        double* eigenvectors, int32_t* iterations, int32_t* status,
                        BatchStats& bs) {
  const int32_t P = static_cast<int32_t>(As.size());
  if (P <= 0) throw Error(FE_ERR_INVALID, "batch: no problems.");
  const std::string which = opt.which;
  if (which != "sr" && which != "lr" && which != "sm" && which != "lm" && which != "be")
    throw Error(FE_ERR_INVALID, "KrylovSchurSolver: invalid which option (use SR/LR/SM/LM/BE/SAI).");
  if (opt.maxiter <= 0) throw Error(FE_ERR_INVALID, "KrylovSchurSolver: maxiter must be > 0.");
  const double tol = opt.tol;
  const int device = As[0]->device;
  std::vector<int64_t> n(P), m(P), row0(P + 1, 0), nz0(P + 1, 0);
  int max_m = 0, max_nev = 0;
  int64_t max_row_nnz = 0;
  for (int32_t p = 0; p < P; ++p) {
    const Csr& A = *As[p];
    FE_REQUIRE(A.device == device, "batch: all problems must live on one device.");
    FE_REQUIRE(A.rows == A.cols && A.rows > 0, "batch: problems must be square and non-empty.");
    n[p] = A.rows;
    if (nevs[p] <= 0 || nevs[p] > n[p])
      throw Error(FE_ERR_INVALID, "KrylovSchurSolver: nev must be in [1,n].");
    m[p] = std::min<int64_t>(std::max<int64_t>({2 * nevs[p], 20, opt.maxdim}), n[p]);
    FE_REQUIRE(m[p] <= kBatchMaxDim, "batch: subspace dimension above " +
                                         std::to_string(kBatchMaxDim) +
                                         " (use the single-problem solver).");
    max_m = std::max<int>(max_m, static_cast<int>(m[p]));
    max_nev = std::max<int>(max_nev, static_cast<int>(nevs[p]));
    max_row_nnz = std::max(max_row_nnz, A.max_row_nnz);
    row0[p + 1] = row0[p] + n[p];
    nz0[p + 1] = nz0[p] + A.nnz;
  }
  const int64_t N = row0[P];
  FE_REQUIRE(N < INT32_MAX && nz0[P] < INT32_MAX, "batch: more than 2^31 rows or nonzeros.");
  const int64_t M = std::max<int64_t>(8, ((max_m + 7) / 8) * 8);
  const int64_t ldy = std::max<int64_t>(8, ((max_nev + 7) / 8) * 8);
  Context ctx;
  cudaStream_t s = ctx.stream;
  // Block-diagonal CSR of all problems.
  DeviceBuffer rp((N + 1) * sizeof(int32_t)), ci(std::max<int64_t>(nz0[P], 1) * sizeof(int32_t)),
      va(std::max<int64_t>(nz0[P], 1) * sizeof(double));
  for (int32_t p = 0; p < P; ++p) {
    const Csr& A = *As[p];
    bks_offset_copy(A.rowptr, n[p], static_cast<int32_t>(nz0[p]), rp.as<int32_t>() + row0[p], s);
    bks_offset_copy(A.colind, A.nnz, static_cast<int32_t>(row0[p]), ci.as<int32_t>() + nz0[p], s);
    if (A.nnz > 0)
      FE_CHECK_CUDA(cudaMemcpyAsync(va.as<double>() + nz0[p], A.val64, A.nnz * sizeof(double),
                                    cudaMemcpyDeviceToDevice, s));
  }
  {
    const int32_t last = static_cast<int32_t>(nz0[P]);
    ctx.to_device(rp.as<int32_t>() + N, &last, 1);
  }
  Csr Aall;
  Aall.rows = Aall.cols = N;
  Aall.nnz = nz0[P];
  Aall.rowptr = rp.as<int32_t>();
  Aall.colind = ci.as<int32_t>();
  Aall.val64 = va.as<double>();
  Aall.device = device;
  Aall.max_row_nnz = max_row_nnz;
  // Reduction chunks.
  std::vector<int32_t> c_prob, c_rows, p_chunk0(P), p_nchunks(P);
  std::vector<int64_t> c_row0;
  for (int32_t p = 0; p < P; ++p) {
    p_chunk0[p] = static_cast<int32_t>(c_prob.size());
    for (int64_t r = 0; r < n[p]; r += kBatchChunkRows) {
      c_prob.push_back(p);
      c_row0.push_back(row0[p] + r);
      c_rows.push_back(static_cast<int32_t>(std::min<int64_t>(kBatchChunkRows, n[p] - r)));
    }
    p_nchunks[p] = static_cast<int32_t>(c_prob.size()) - p_chunk0[p];
  }
  const int32_t NC = static_cast<int32_t>(c_prob.size());
  DeviceBuffer d_cprob(NC * 4), d_crow0(NC * 8), d_crows(NC * 4), d_pc0(P * 4), d_pnc(P * 4);
  ctx.to_device(d_cprob.as<int32_t>(), c_prob.data(), NC);
  ctx.to_device(d_crow0.as<int64_t>(), c_row0.data(), NC);
  ctx.to_device(d_crows.as<int32_t>(), c_rows.data(), NC);
  ctx.to_device(d_pc0.as<int32_t>(), p_chunk0.data(), P);
  ctx.to_device(d_pnc.as<int32_t>(), p_nchunks.data(), P);
  BatchLayout L;
  L.num_problems = P;
  L.num_chunks = NC;
  L.M = M;
  L.c_prob = d_cprob.as<int32_t>();
  L.c_row0 = d_crow0.as<int64_t>();
  L.c_rows = d_crows.as<int32_t>();
  L.p_chunk0 = d_pc0.as<int32_t>();
  L.p_nchunks = d_pnc.as<int32_t>();
  // Blocks and per-problem state.
  DeviceBuffer V(static_cast<size_t>(N) * M * 8), f(N * 8), q(N * 8), w(N * 8);
  DeviceBuffer d_col(P * 4), d_m(P * 4), d_rr(P * 4), d_act(P * 4), d_status(P * 4), d_beta(P * 8),
      d_inv(P * 8), d_bn(P * 8), d_T(static_cast<size_t>(P) * M * M * 8),
      d_part(static_cast<size_t>(NC) * M * 8), d_part1(NC * 8), d_h1(P * M * 8), d_h2(P * M * 8),
      d_W(P * M * 8), d_Z(static_cast<size_t>(P) * M * M * 8), d_C(static_cast<size_t>(P) * M * M * 8),
      d_todo(P * 4), d_keep(P * 4), d_keepY(P * 4), d_Zl(P * M * 8), d_idx(P * M * 4),
      d_diag(P * M * 8), d_coup(P * M * 8);
  BatchState S;
  S.col = d_col.as<int32_t>();
  S.mdim = d_m.as<int32_t>();
  S.restart_row = d_rr.as<int32_t>();
  S.active = d_act.as<int32_t>();
  S.status = d_status.as<int32_t>();
  S.beta = d_beta.as<double>();
  S.inv = d_inv.as<double>();
  S.beta_next = d_bn.as<double>();
  S.T = d_T.as<double>();
  S.part = d_part.as<double>();
  S.part1 = d_part1.as<double>();
  S.h1 = d_h1.as<double>();
  S.h2 = d_h2.as<double>();
  std::vector<int32_t> h_col(P, 0), h_m(P), h_rr(P, -1), h_act(P, 1), h_status(P, 0);
  for (int32_t p = 0; p < P; ++p) h_m[p] = static_cast<int32_t>(m[p]);
  auto upload_state = [&] {
    ctx.to_device(S.col, h_col.data(), P);
    ctx.to_device(S.restart_row, h_rr.data(), P);
    ctx.to_device(S.active, h_act.data(), P);
  };
  ctx.to_device(S.mdim, h_m.data(), P);
  ctx.to_device(S.status, h_status.data(), P);
  FE_CHECK_CUDA(cudaMemsetAsync(S.T, 0, d_T.bytes(), s));
  upload_state();
  // Starting vectors: each problem's own seeded draw (the single solver's
  // random_into(f, seed)), so a problem starts identically alone or batched.
  const unsigned seed = opt.seed_or_default();
  if (opt.init == "host") {
    std::vector<double> hf(N);
    for (int32_t p = 0; p < P; ++p) {
      std::mt19937 rng(seed);
      std::uniform_real_distribution<double> dist(-1.0, 1.0);
      for (int64_t i = 0; i < n[p]; ++i) hf[row0[p] + i] = dist(rng);
    }
    ctx.to_device(f.as<double>(), hf.data(), N);
  } else {
    for (int32_t p = 0; p < P; ++p) fill_uniform<double>(f.as<double>() + row0[p], 1, n[p], 1, seed, s);
  }
  FE_CHECK_CUDA(cudaMemsetAsync(V.get(), 0, V.bytes(), s));
  bks_init_norm(L, S, f.as<double>(), s);
  ctx.sync();
  // One Lanczos step of the whole batch as a CUDA graph.
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  FE_CHECK_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  try {
    bks_lanczos_step(L, S, Aall, V.as<double>(), M, f.as<double>(), q.as<double>(), w.as<double>(), s);
  } catch (...) {
    cudaStreamEndCapture(s, &graph);
    if (graph) cudaGraphDestroy(graph);
    throw;
  }
  FE_CHECK_CUDA(cudaStreamEndCapture(s, &graph));
  struct GraphGuard {
    cudaGraph_t g;
    cudaGraphExec_t* e;
    ~GraphGuard() {
      if (*e) cudaGraphExecDestroy(*e);
      if (g) cudaGraphDestroy(g);
    }
  } guard{graph, &exec};
  FE_CHECK_CUDA(cudaGraphInstantiate(&exec, graph, 0));

  const auto t0 = std::chrono::steady_clock::now();
  std::vector<char> finished(P, 0);
  std::vector<double> lam_final(static_cast<size_t>(P) * ldy, 0.0);
  std::vector<int32_t> keep(P, 0), keepY(P, 0), todo(P, 0), nev32(P);
  for (int32_t p = 0; p < P; ++p) nev32[p] = static_cast<int32_t>(nevs[p]);
  std::vector<double> hW(static_cast<size_t>(P) * M), hZl(static_cast<size_t>(P) * M),
      hdiag(static_cast<size_t>(P) * M, 0.0), hcoup(static_cast<size_t>(P) * M, 0.0), hbn(P);
  std::vector<int32_t> hidx(static_cast<size_t>(P) * M, 0);
  DeviceBuffer Y(static_cast<size_t>(N) * ldy * 8);
  FE_CHECK_CUDA(cudaMemsetAsync(Y.get(), 0, Y.bytes(), s));
  int64_t steps_needed = max_m;
  for (int64_t iter = 1;; ++iter) {
    for (int64_t k = 0; k < steps_needed; ++k) FE_CHECK_CUDA(cudaGraphLaunch(exec, s));
    bs.steps += static_cast<double>(steps_needed);
    bs.graph_launches += static_cast<double>(steps_needed);
    bs.rounds += 1;
    ctx.to_host(h_status.data(), S.status, P);
    ctx.sync();
    for (int32_t p = 0; p < P; ++p) {
      if (finished[p]) continue;
      if (h_status[p] == 2)
        throw Error(FE_ERR_NONFINITE,
                    "core::KrylovSubspace: breakdown in batched problem " + std::to_string(p) +
                        " (solve it alone for the randomized restart).");
      if (h_status[p] != 0)
        throw Error(FE_ERR_NONFINITE, "core::KrylovSubspace: non-finite residual norm encountered.");
      todo[p] = 1;
    }
    ctx.to_device(d_todo.as<int32_t>(), todo.data(), P);
    bks_jacobi(L, S.T, S.mdim, d_todo.as<int32_t>(), max_m, d_W.as<double>(), d_Z.as<double>(),
               d_Zl.as<double>(), s);
    ctx.to_host(hW.data(), d_W.as<double>(), hW.size());
    ctx.to_host(hZl.data(), d_Zl.as<double>(), hZl.size());
    ctx.to_host(hbn.data(), S.beta_next, P);
    ctx.sync();
    int max_keep = 0, max_keepY = 0;
    bool any_active = false;
    for (int32_t p = 0; p < P; ++p) {
      keep[p] = keepY[p] = 0;
      h_act[p] = 0;
      if (finished[p]) continue;
      todo[p] = 0;
      const int64_t mp = m[p], nev = nevs[p];
      std::vector<double> lam(hW.begin() + static_cast<int64_t>(p) * M,
                              hW.begin() + static_cast<int64_t>(p) * M + mp);
      const double* Zl = hZl.data() + static_cast<size_t>(p) * M;  // last row of Z_p
      const std::vector<int32_t> idx = select_indices(lam, which);
      std::copy(idx.begin(), idx.end(), hidx.begin() + static_cast<size_t>(p) * M);
      std::vector<double> lam_s(mp), rel_s(mp);
      for (int64_t j = 0; j < mp; ++j) {
        lam_s[j] = lam[idx[j]];
        rel_s[j] = std::fabs(hbn[p] * Zl[idx[j]]) / (1.0 + std::fabs(lam_s[j]));
      }
      int64_t nconv = 0;
      for (int64_t j = 0; j < nev; ++j) {
        const double mag = std::fabs(lam_s[j]);
        if (rel_s[j] * (1.0 + mag) < tol * mag) ++nconv;
      }
      const bool at_limit = (mp == n[p]) || (iter == opt.maxiter);
      if (nconv >= nev || at_limit) {
        for (int64_t j = 0; j < nev; ++j) lam_final[static_cast<size_t>(p) * ldy + j] = lam_s[j];
        keepY[p] = static_cast<int32_t>(nev);
        max_keepY = std::max<int>(max_keepY, static_cast<int>(nev));
        iterations[p] = static_cast<int32_t>(iter);
        status[p] = 0;
        finished[p] = 1;
        continue;
      }
      const int64_t spare = (mp - nev) / 2;
      int64_t retained = nev + std::min(nconv, spare);
      if (retained == 1 && mp > 3) retained = mp / 2;
      keep[p] = static_cast<int32_t>(retained);
      max_keep = std::max<int>(max_keep, static_cast<int>(retained));
      for (int64_t j = 0; j < retained; ++j) {
        hdiag[static_cast<size_t>(p) * M + j] = lam_s[j];
        hcoup[static_cast<size_t>(p) * M + j] = hbn[p] * Zl[idx[j]];
      }
      h_col[p] = static_cast<int32_t>(retained);
      h_rr[p] = static_cast<int32_t>(retained);
      h_act[p] = 1;
      any_active = true;
    }
    ctx.to_device(d_idx.as<int32_t>(), hidx.data(), hidx.size());
    ctx.to_device(d_keep.as<int32_t>(), keep.data(), P);
    ctx.to_device(d_keepY.as<int32_t>(), keepY.data(), P);
    ctx.to_device(d_diag.as<double>(), hdiag.data(), hdiag.size());
    ctx.to_device(d_coup.as<double>(), hcoup.data(), hcoup.size());
    // Coefficients and the restarted T on the device; then finishing problems'
    // Ritz vectors into Y and restarting problems' V[:, :retained] = V C.
    bks_restart(L, S.mdim, d_idx.as<int32_t>(), d_keep.as<int32_t>(), d_keepY.as<int32_t>(),
                d_diag.as<double>(), d_coup.as<double>(), d_Z.as<double>(), d_C.as<double>(), S.T,
                s);
    bks_rotate(L, V.as<double>(), M, d_C.as<double>(), S.mdim, d_keepY.as<int32_t>(), max_m,
               max_keepY, Y.as<double>(), ldy, s);
    bks_rotate(L, V.as<double>(), M, d_C.as<double>(), S.mdim, d_keep.as<int32_t>(), max_m,
               max_keep, V.as<double>(), M, s);
    if (!any_active) break;
    upload_state();
    steps_needed = 0;
    for (int32_t p = 0; p < P; ++p)
      if (h_act[p]) steps_needed = std::max<int64_t>(steps_needed, m[p] - h_col[p]);
  }
  // Final Ritz residuals on the device (evaluate_ritz_pairs, src/core/RitzExtraction.cpp:34-63).
  DeviceBuffer AY(static_cast<size_t>(N) * ldy * 8), d_lam(static_cast<size_t>(P) * ldy * 8),
      d_rel(static_cast<size_t>(P) * ldy * 8), d_nev(P * 4),
      d_rpart(static_cast<size_t>(NC) * 2 * ldy * 8);
  ctx.to_device(d_lam.as<double>(), lam_final.data(), lam_final.size());
  ctx.to_device(d_nev.as<int32_t>(), nev32.data(), P);
  csr_spmm<double>(Aall, Y.as<double>(), ldy, AY.as<double>(), ldy, nullptr, 0, max_nev, 1.0, 0.0,
                   0.0, s);
  bks_residuals(L, d_nev.as<int32_t>(), AY.as<double>(), Y.as<double>(), ldy, d_lam.as<double>(),
                static_cast<int>(ldy), d_rpart.as<double>(), d_rel.as<double>(), s);
  std::vector<double> rel(static_cast<size_t>(P) * ldy);
  ctx.to_host(rel.data(), d_rel.as<double>(), rel.size());
  std::vector<double> hY;
  if (eigenvectors) {
    hY.resize(static_cast<size_t>(N) * ldy);
    ctx.to_host(hY.data(), Y.as<double>(), hY.size());
  }
  ctx.sync();
  bs.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  int64_t off = 0, voff = 0;
  for (int32_t p = 0; p < P; ++p) {
    for (int64_t j = 0; j < nevs[p]; ++j) {
      eigenvalues[off + j] = lam_final[static_cast<size_t>(p) * ldy + j];
      residuals[off + j] = rel[static_cast<size_t>(p) * ldy + j];
      if (!std::isfinite(residuals[off + j]))
        throw Error(FE_ERR_NONFINITE, "evaluate_ritz_pairs: invalid vector or non-finite residual.");
    }
    if (eigenvectors) {
      for (int64_t j = 0; j < nevs[p]; ++j)
        for (int64_t i = 0; i < n[p]; ++i)
          eigenvectors[voff + j * n[p] + i] = hY[static_cast<size_t>(row0[p] + i) * ldy + j];
      voff += n[p] * nevs[p];
    }
    off += nevs[p];
  }
}

}  // namespace
}  // namespace fe

namespace fe {

// Solver dispatch of fasteig_problem::solve (src/fasteig_problem.cpp:340-437) on
// device CSR operators; throws fe::Error. Shared by fe_solve and the request server.
void solve_problem(const Csr& A, const Csr* B, const char* options, double* eigenvalues,
                   double* residual_norms, double* eigenvectors, double* stats) {
  FE_REQUIRE(eigenvalues && residual_norms, "null result arrays");
  Options opt;
  opt.parse(options);
  Stats st;
  const auto t0 = std::chrono::steady_clock::now();
  FE_CHECK_CUDA(cudaSetDevice(A.device));
  // This solve's own device status word: a bounded wait that runs out in one of its
  // kernels is reported here, to this solve, and not to whichever solve reads the
  // library's default word next.
  int32_t* status_word = thread_status_word();
  FE_CHECK_CUDA(cudaMemset(status_word, 0, sizeof(int32_t)));
  StatusScope status_scope(status_word);
  if (opt.inject_wait_timeout != 0) {
    // Test hook: a probe kernel whose bounded wait runs out (about a millisecond of
    // SM clock on an mbarrier nothing arrives on) records the code in this solve's
    // word, as a real timeout in a solve kernel would.
    launch_wait_probe(status_word, 2000000LL, static_cast<int>(opt.inject_wait_timeout),
                      nullptr);
    FE_CHECK_CUDA(cudaStreamSynchronize(nullptr));
  }
  if (opt.solver == "chebyshev") {
    FE_REQUIRE(B == nullptr, "ChebyshevSolver: generalized problems are not supported.");
    chebyshev_solve(A, opt, eigenvalues, residual_norms, eigenvectors, st);
  } else if (opt.solver == "lobpcg") {
    // The reference's standard unpreconditioned LOBPCG unless the problem is
    // generalized, preconditioned, or iterates more vectors than requested.
    if (B || opt.precond != "none" || opt.block > opt.nev || opt.precision == "mixed") {
      if (B) check_pair(A, *B);
      lobpcg_gen_solve(A, B, opt, eigenvalues, residual_norms, eigenvectors, st);
    } else {
      lobpcg_solve(A, opt, eigenvalues, residual_norms, eigenvectors, st);
    }
  } else if (opt.solver == "davidson") {
    if (B || opt.precond != "none" || opt.block > opt.nev || opt.precision == "mixed") {
      if (B) check_pair(A, *B);
      davidson_gen_solve(A, B, opt, eigenvalues, residual_norms, eigenvectors, st);
    } else {
      davidson_solve(A, opt, eigenvalues, residual_norms, eigenvectors, st);
    }
  } else if (opt.solver == "blockkrylovschur") {
    FE_REQUIRE(B == nullptr,
               "BlockKrylovSchurSolver: generalized problems are not supported on this backend.");
    block_krylov_schur_solve(A, opt, eigenvalues, residual_norms, eigenvectors, st);
  } else if (opt.solver == "krylovschur") {
    if (B) check_pair(A, *B);
    krylov_schur_solve(A, B, opt, eigenvalues, residual_norms, eigenvectors, st);
  } else if (opt.solver == "lanczos") {
    if (B) check_pair(A, *B);
    lanczos_solve(A, B, opt, eigenvalues, residual_norms, eigenvectors, st);
  } else {
    throw Error(FE_ERR_UNSUPPORTED, "solver not available on this backend: " + opt.solver);
  }
  int32_t word = 0;
  FE_CHECK_CUDA(cudaMemcpy(&word, status_word, sizeof(int32_t), cudaMemcpyDeviceToHost));
  if (word != 0)
    throw Error(FE_ERR_CUDA, "device wait timed out in a solve kernel (status code " +
                                 std::to_string(word) + "); results discarded");
  const auto t1 = std::chrono::steady_clock::now();
  st.seconds = std::chrono::duration<double>(t1 - t0).count();
  if (opt.verbosity >= 2)
    std::fprintf(stderr, "[fe] solve total (incl. buffer release) %.1f ms\n", st.seconds * 1e3);
  if (stats) {
    stats[0] = st.iterations;
    stats[1] = st.status;
    stats[2] = st.seconds;
    stats[3] = st.spmm_launches;
    stats[4] = st.fp32_iterations;
    stats[5] = st.fp64_iterations;
    stats[6] = st.lower;
    stats[7] = st.upper;
    stats[8] = st.filter_ms;
    stats[9] = st.ortho_ms;
    stats[10] = st.rr_ms;
    stats[11] = st.precise_grams;
  }
}

// ---------------------------------------------------------------------------
// Grouped Chebyshev members (grouped.cpp runs them): which requests may join a
// group, and the per-problem setup the reference's ChebyshevSolver does before its
// loop (src/ChebyshevSolver.cpp:67-129): option checks, the subspace width, and the
// Lanczos spectral bounds (estimate_bounds_with_executor, :26-49).
// ---------------------------------------------------------------------------

// Subspace width of a grouped member: the solve's capacity (nev + min(nev, n - nev),
// or `block`), rounded up to a multiple of 32 (members of one width share a group).
static int64_t group_width_of(const Options& opt, int64_t n) {
  int64_t cap = opt.nev + std::min(opt.nev, n - opt.nev);
  if (opt.block > 0) cap = std::max(opt.nev, std::min(opt.block, n));
  return (cap + 31) / 32 * 32;
}

bool chebyshev_group_key(const Csr& A, const Csr* B, const char* options, bool require_flag,
                         int64_t* width, int64_t* degree, bool* mixed) {
  Options opt;
  opt.parse(options);
  if (require_flag && !opt.group) return false;
  if (opt.solver != "chebyshev" || B != nullptr || A.rows != A.cols) return false;
  if ((opt.precision != "fp64" && opt.precision != "mixed") || opt.locking != "soft") return false;
  if (opt.which != "sr" && opt.which != "lr") return false;
  if (opt.nev < 1 || opt.nev > A.rows || opt.degree < 1) return false;
  const int64_t w = group_width_of(opt, A.rows);
  if (w > A.rows || w > 512) return false;
  if (width) *width = w;
  if (degree) *degree = opt.degree;
  if (mixed) *mixed = opt.precision == "mixed";
  return true;
}

void chebyshev_group_setup(const Csr& A, const char* options, GroupSetup& g) {
  Options opt;
  opt.parse(options);
  FE_REQUIRE(chebyshev_group_key(A, nullptr, options, false, nullptr, nullptr),
             "grouped Chebyshev: request not eligible (standard FP64 or mixed Chebyshev with "
             "soft locking and a width of at most 512 columns)");
  FE_REQUIRE(opt.bounds == "reference" || opt.bounds == "ritz", "bounds must be reference or ritz");
  FE_REQUIRE(opt.init == "host" || opt.init == "device", "init must be host or device");
  g.n = A.rows;
  g.nev = opt.nev;
  g.width = group_width_of(opt, A.rows);
  g.degree = opt.degree;
  g.maxiter = opt.maxiter;
  g.tol = opt.tol;
  g.sign = opt.which == "lr" ? -1.0 : 1.0;
  g.seed = opt.seed_or_default();
  g.host_init = opt.init == "host";
  g.ritz_bounds = opt.bounds == "ritz";
  g.amplification = opt.amplification;
  g.mixed = opt.precision == "mixed";
  g.mixed_switch = opt.mixed_switch;
  Context ctx;
  {
    // the filter operator c A + d I is written into each row's stored diagonal
    DeviceBuffer bad(sizeof(int32_t));
    csr_count_bad_diagonals(A, bad.as<int32_t>(), ctx.stream);
    int32_t nbad = 0;
    ctx.to_host(&nbad, bad.as<int32_t>(), 1);
    ctx.sync();
    FE_REQUIRE(nbad == 0, "grouped Chebyshev: every row needs exactly one stored diagonal "
                          "entry (" + std::to_string(nbad) + " rows without)");
  }
  lanczos_bounds(ctx, A, g.sign, g.seed, g.host_init, g.lower, g.upper);
  g.reference_cutoff = reference_cutoff(g.lower, g.upper, g.degree, 1.0e3);
  g.ritz_cutoff_cap = reference_cutoff(g.lower, g.upper, g.degree, g.amplification);
}

// nev of an option string, validating every key as the solve will.
int64_t options_nev(const char* options) {
  Options opt;
  opt.parse(options);
  return opt.nev;
}

// Upper bound of the device memory one solve allocates (its blocks and
// workspaces; the CSR operators are the caller's), for admission control.
size_t solve_memory_bytes(const Csr& A, const Csr* B, const char* options) {
  Options opt;
  opt.parse(options);
  const int64_t n = A.rows;
  const int64_t nev = std::max<int64_t>(1, std::min<int64_t>(opt.nev, n));
  auto ld = [](int64_t c) { return std::max<int64_t>(8, ((c + 7) / 8) * 8); };
  double blocks = 0;  // n x ld doubles
  int64_t cap = nev;
  if (opt.solver == "chebyshev") {
    cap = nev + std::min(nev, n - nev);
    if (opt.block > 0) cap = std::max(nev, std::min(opt.block, n));
    // FP64: 4 loop blocks + 2 initial; mixed adds 4 FP32 blocks (half size), the
    // refined filter's 3 FP32 blocks and the widened copy of an FP32 block that an
    // FP64-accumulated Gram retry allocates for its duration.
    blocks = opt.precision == "mixed" ? 4 + 2 + 2 + 1.5 + 1 + 1 : 4 + 2 + 1;
  } else if (opt.solver == "lobpcg") {
    cap = std::min<int64_t>(n, 3 * std::max<int64_t>(nev, opt.block));
    blocks = 12;
  } else if (opt.solver == "davidson") {
    cap = std::min<int64_t>(n, opt.maxblks * std::max<int64_t>(nev, opt.block));
    blocks = 11;
  } else if (opt.solver == "blockkrylovschur") {
    const int64_t b = std::max<int64_t>(1, opt.blksize);
    cap = std::min<int64_t>(opt.maxdim > 0 ? opt.maxdim : std::max<int64_t>(2 * nev, 20), n) + b;
    blocks = 2 + 5.0 * static_cast<double>(b) / static_cast<double>(cap);
  } else {
    cap = std::min<int64_t>(std::max<int64_t>({2 * nev, 20, opt.maxdim}), n);
    blocks = 3;
  }
  (void)B;
  // Workspaces: Gram partials (the split-TF32 Gram's per-chunk tiles dominate),
  // residual sums, rotation operands, the eigensolver, the multi-step filter's
  // counters, the k x k FP64 matrices, and slack for small buffers.
  const size_t gram_ws = std::max(gram_workspace_bytes(n, cap, cap),
                                  tc_gram_workspace_bytes(n, cap, cap));
  const double ws = static_cast<double>(gram_ws) +
                    static_cast<double>(residual_workspace_bytes(n, cap)) +
                    static_cast<double>(tc_rotate_workspace_bytes(cap, cap)) +
                    static_cast<double>(syevd_single_workspace_bytes(cap)) +
                    static_cast<double>(wave_sync_bytes(n)) +
                    16.0 * static_cast<double>(cap) * cap * 8.0 + (64u << 20);
  const double bytes = blocks * static_cast<double>(n) * ld(cap) * 8.0 + ws;
  return static_cast<size_t>(bytes);
}

}  // namespace fe

extern "C" int fe_solve(fe_csr_t A, fe_csr_t B, const char* options, double* eigenvalues,
                        double* residual_norms, double* eigenvectors, double* stats) {
  return fe::guarded("fe_solve", [&] {
    FE_REQUIRE(A, "null CSR handle");
    fe::solve_problem(A->m, B ? &B->m : nullptr, options, eigenvalues, residual_norms,
                      eigenvectors, stats);
  });
}

extern "C" int fe_batch_krylov_schur(int32_t count, const fe_csr_t* A, const int64_t* nev,
                                     const char* options, double* eigenvalues,
                                     double* residual_norms, double* eigenvectors,
                                     int32_t* iterations, int32_t* status, double* stats) {
  return fe::guarded("fe_batch_krylov_schur", [&] {
    FE_REQUIRE(count > 0 && A && nev, "null or empty batch");
    FE_REQUIRE(eigenvalues && residual_norms && iterations && status, "null result arrays");
    fe::Options opt;
    opt.parse(options);
    std::vector<const fe::Csr*> As(count);
    std::vector<int64_t> nevs(nev, nev + count);
    for (int32_t p = 0; p < count; ++p) {
      FE_REQUIRE(A[p], "null CSR handle in batch");
      As[p] = &A[p]->m;
    }
    FE_CHECK_CUDA(cudaSetDevice(As[0]->device));
    fe::BatchStats bs;
    fe::batch_krylov_schur(As, nevs, opt, eigenvalues, residual_norms, eigenvectors, iterations,
                           status, bs);
    if (stats) {
      stats[0] = bs.seconds;
      stats[1] = bs.rounds;
      stats[2] = bs.steps;
      stats[3] = bs.graph_launches;
    }
  });
}
