// The fe_solve branch a fasteig maintainer adds to fasteig_problem::solve
// (src/fasteig_problem.cpp:340-437), compiled against minimal stand-ins of the
// reference types it touches: fasteig_options' typed accessors
// (include/fasteig_options.hpp:41-62), CsrMatrixData (include/core/CsrMatrix.hpp:18-27)
// and the problem's result members (include/fasteig_problem.hpp:48-56,145-184). Eigen
// is not installed here, so VectorXd / MatrixXd are column-major stand-ins with the
// same data layout.
//
// Usage: fasteig_adapter <input> <solver> [<solver> ...] (input layout as consumer.c).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <iomanip>
#include <optional>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "fasteig_b200.h"

using FASTEIG_INT = long long;

struct VectorXd {
  std::vector<double> v;
  void resize(FASTEIG_INT n) { v.assign(static_cast<size_t>(n), 0.0); }
  double* data() { return v.data(); }
  double operator[](FASTEIG_INT i) const { return v[static_cast<size_t>(i)]; }
};

struct MatrixXd {  // column-major, like Eigen's default
  FASTEIG_INT r = 0, c = 0;
  std::vector<double> v;
  void resize(FASTEIG_INT rows, FASTEIG_INT cols) {
    r = rows;
    c = cols;
    v.assign(static_cast<size_t>(rows * cols), 0.0);
  }
  double* data() { return v.data(); }
  double operator()(FASTEIG_INT i, FASTEIG_INT j) const { return v[static_cast<size_t>(j * r + i)]; }
};

struct CsrMatrixData {
  FASTEIG_INT rows = 0, cols = 0;
  std::vector<int> rowptr, colind;
  std::vector<double> values;
};

class fasteig_options {
 public:
  FASTEIG_INT nev_ = 10, maxiter_ = 1000, maxdim_ = 0, maxblks_ = 10, degree_ = 10;
  std::string which_ = "LM";
  double tol_ = 1e-8;
  std::optional<unsigned int> seed_;
  bool gpu_backend_ = false;
  FASTEIG_INT nev() const noexcept { return nev_; }
  FASTEIG_INT maxiter() const noexcept { return maxiter_; }
  FASTEIG_INT maxdim() const noexcept { return maxdim_; }
  FASTEIG_INT maxblks() const noexcept { return maxblks_; }
  FASTEIG_INT degree() const noexcept { return degree_; }
  const std::string& which() const noexcept { return which_; }
  double tol() const noexcept { return tol_; }
  std::optional<unsigned int> seed() const noexcept { return seed_; }
  bool gpu_backend() const noexcept { return gpu_backend_; }
};

class fasteig_problem {
 public:
  explicit fasteig_problem(CsrMatrixData A) : n_(A.rows), csrA_(std::move(A)) {}
  // The reference's FASTEIG_INT solve(const fasteig_options&) returns the solver
  // status; this stand-in has no reference path behind the B200 branch and throws
  // std::logic_error when the branch does not take the solve.
  FASTEIG_INT solve(const fasteig_options& local, const std::string& solver_name);
  VectorXd eigvals_, resnrms_;
  MatrixXd eigvecs_;
  FASTEIG_INT status_ = 0;
  std::optional<long long> last_iterations_;

 private:
  FASTEIG_INT n_ = 0;
  std::optional<CsrMatrixData> csrA_;
  std::optional<CsrMatrixData> B_;
};

FASTEIG_INT fasteig_problem::solve(const fasteig_options& local, const std::string& solver_name) {
  eigvals_.resize(local.nev());
  resnrms_.resize(local.nev());
  // BEGIN fe_solve branch
  static const std::set<std::string> on_b200 = {"Chebyshev", "LOBPCG", "Davidson",
                                                 "KrylovSchur"};
  if (local.gpu_backend() && csrA_ && on_b200.count(solver_name) && !B_) {
    fe_csr_t A = nullptr;
    if (fe_csr_create(n_, n_, static_cast<int64_t>(csrA_->values.size()), csrA_->rowptr.data(),
                      csrA_->colind.data(), csrA_->values.data(), &A) != FE_OK)
      throw std::runtime_error(fe_last_error());
    std::ostringstream o;
    o << "solver=" << solver_name << "\nnev=" << local.nev() << "\nmaxiter=" << local.maxiter()
      << "\nmaxdim=" << local.maxdim() << "\nmaxblks=" << local.maxblks()
      << "\ndegree=" << local.degree() << "\nwhich=" << local.which()
      << "\ntol=" << std::setprecision(17) << local.tol();
    if (local.seed()) o << "\nseed=" << *local.seed();
    double stats[12];
    eigvecs_.resize(n_, local.nev());  // column-major n x nev, like Eigen
    const int rc = fe_solve(A, nullptr, o.str().c_str(), eigvals_.data(), resnrms_.data(),
                            eigvecs_.data(), stats);
    fe_csr_destroy(A);
    if (rc == FE_ERR_INVALID) throw std::invalid_argument(fe_last_error());
    if (rc != FE_OK) throw std::runtime_error(fe_last_error());
    status_ = static_cast<FASTEIG_INT>(stats[1]);
    last_iterations_ = static_cast<long long>(stats[0]);
    // resnrms_ already holds the FP64 final residual check of the returned pairs.
    return status_;
  }
  // END fe_solve branch
  throw std::logic_error("not a B200 solve: the reference path is not part of this stand-in");
}

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 2;
  int64_t hdr[3];
  if (std::fread(hdr, sizeof(int64_t), 3, f) != 3) return 3;
  CsrMatrixData A;
  A.rows = A.cols = hdr[0];
  A.rowptr.resize(static_cast<size_t>(hdr[0] + 1));
  A.colind.resize(static_cast<size_t>(hdr[1]));
  A.values.resize(static_cast<size_t>(hdr[1]));
  std::vector<double> expected(static_cast<size_t>(hdr[2]));
  bool ok = std::fread(A.rowptr.data(), sizeof(int), A.rowptr.size(), f) == A.rowptr.size() &&
            std::fread(A.colind.data(), sizeof(int), A.colind.size(), f) == A.colind.size() &&
            std::fread(A.values.data(), sizeof(double), A.values.size(), f) == A.values.size() &&
            std::fread(expected.data(), sizeof(double), expected.size(), f) == expected.size();
  std::fclose(f);
  if (!ok) return 3;
  fasteig_problem prob(A);
  int failures = 0;
  // An invalid option value surfaces as the reference's exception type.
  {
    fasteig_options bad;
    bad.gpu_backend_ = true;
    bad.nev_ = 0;
    bad.which_ = "SR";
    try {
      prob.solve(bad, "Chebyshev");
      std::fprintf(stderr, "nev=0 accepted\n");
      ++failures;
    } catch (const std::invalid_argument&) {
    }
  }
  for (int s = 2; s < argc; ++s) {
    fasteig_options opts;
    opts.gpu_backend_ = true;
    opts.nev_ = static_cast<FASTEIG_INT>(expected.size());
    opts.maxiter_ = 3000;
    opts.which_ = "SR";
    opts.seed_ = 1u;
    try {
      if (prob.solve(opts, argv[s]) != 0) {
        std::fprintf(stderr, "%s: status %lld\n", argv[s], prob.status_);
        ++failures;
      }
    } catch (const std::logic_error& e) {
      std::fprintf(stderr, "%s: %s\n", argv[s], e.what());
      ++failures;
      continue;
    }
    for (size_t j = 0; j < expected.size(); ++j) {
      const double l = prob.eigvals_[static_cast<FASTEIG_INT>(j)];
      if (!(std::fabs(l - expected[j]) <= 1e-10 + 1e-10 * std::fabs(expected[j])) ||
          !(prob.resnrms_[static_cast<FASTEIG_INT>(j)] <= 1e-8)) {
        std::fprintf(stderr, "%s pair %zu: %.15g vs %.15g\n", argv[s], j, l, expected[j]);
        ++failures;
      }
    }
    std::printf("%s: status %lld, %lld iterations, lowest %.12f\n", argv[s], prob.status_,
                prob.last_iterations_.value_or(-1), prob.eigvals_[0]);
  }
  return failures ? 1 : 0;
}
