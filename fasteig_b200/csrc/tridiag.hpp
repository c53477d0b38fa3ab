// Selected eigenpairs of a symmetric tridiagonal matrix on the host: the projected
// matrix of a Lanczos chain (diagonal d[0..m), off-diagonal e[0..m-1), e[i] = T(i+1, i)).
// Eigenvalues by bisection on Sturm counts (only those the selection can need, so a
// snapshot of a long chain costs O(m * nev) per bisection step), eigenvectors by
// inverse iteration on T - theta I (LU with partial pivoting) with the vectors of a
// cluster reorthogonalized, as LAPACK's stebz/stein divide the work. Host only, no
// CUDA dependency.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <string>
#include <vector>

namespace fe {

struct TridiagEig {
  const std::vector<double>& d;
  const std::vector<double>& e;
  int m;
  double tnorm = 0.0, pivmin = 0.0, lo = 0.0, hi = 0.0;
  std::vector<double> e2;

  TridiagEig(const std::vector<double>& d_, const std::vector<double>& e_, int m_)
      : d(d_), e(e_), m(m_) {
    e2.resize(std::max(m - 1, 0));
    lo = std::numeric_limits<double>::infinity();
    hi = -lo;
    double emax = 0.0;
    for (int i = 0; i < m; ++i) {
      const double left = i > 0 ? std::fabs(e[i - 1]) : 0.0;
      const double right = i < m - 1 ? std::fabs(e[i]) : 0.0;
      lo = std::min(lo, d[i] - left - right);
      hi = std::max(hi, d[i] + left + right);
      tnorm = std::max(tnorm, std::fabs(d[i]) + left + right);
      if (i < m - 1) {
        e2[i] = e[i] * e[i];
        emax = std::max(emax, e2[i]);
      }
    }
    pivmin = std::numeric_limits<double>::min() * std::max(1.0, emax);
    const double pad = 2.0 * std::numeric_limits<double>::epsilon() * tnorm + pivmin;
    lo -= pad;
    hi += pad;
  }

  // Number of eigenvalues below x (negative pivots of the LDL^T of T - x I).
  int count_below(double x) const {
    int cnt = 0;
    double q = d[0] - x;
    if (std::fabs(q) < pivmin) q = -pivmin;
    cnt += q < 0.0;
    for (int i = 1; i < m; ++i) {
      q = d[i] - x - e2[i - 1] / q;
      if (std::fabs(q) < pivmin) q = -pivmin;
      cnt += q < 0.0;
    }
    return cnt;
  }

  // The j-th smallest eigenvalue (0-based), by bisection to rounding level.
  double eigenvalue(int j) const {
    double a = lo, b = hi;
    const double atol = 2.0 * std::numeric_limits<double>::epsilon();
    for (int it = 0; it < 200; ++it) {
      const double mid = 0.5 * (a + b);
      if (b - a <= atol * std::max(std::fabs(a), std::fabs(b)) + pivmin || mid == a || mid == b)
        break;
      if (count_below(mid) > j) b = mid;
      else a = mid;
    }
    return 0.5 * (a + b);
  }

  // Unit eigenvector of eigenvalue theta by inverse iteration (three solves with
  // T - theta I factored once), orthogonalized after every solve against the given
  // vectors (the already computed members of its cluster).
  std::vector<double> vector(double theta, unsigned seed,
                             const std::vector<const std::vector<double>*>& against) const {
    std::vector<double> u0(m), u1(m, 0.0), u2(m, 0.0), l(m, 0.0);
    std::vector<char> piv(m, 0);
    const double tiny = std::numeric_limits<double>::epsilon() * std::max(tnorm, pivmin);
    u0[0] = d[0] - theta;
    if (m > 1) u1[0] = e[0];
    for (int i = 0; i + 1 < m; ++i) {
      const double sub = e[i];
      const double a1 = d[i + 1] - theta;
      const double e1 = i + 2 < m ? e[i + 1] : 0.0;
      if (std::fabs(sub) > std::fabs(u0[i])) {
        // swap rows i and i + 1, then eliminate the old row i
        const double mult = u0[i] / sub;
        const double r1 = u1[i] - mult * a1;
        const double r2 = u2[i] - mult * e1;
        u0[i] = sub;
        u1[i] = a1;
        u2[i] = e1;
        u0[i + 1] = r1;
        u1[i + 1] = r2;
        l[i] = mult;
        piv[i] = 1;
      } else {
        const double mult = u0[i] != 0.0 ? sub / u0[i] : 0.0;
        u0[i + 1] = a1 - mult * u1[i];
        u1[i + 1] = e1 - mult * u2[i];
        l[i] = mult;
      }
    }
    for (int i = 0; i < m; ++i)
      if (std::fabs(u0[i]) < tiny) u0[i] = u0[i] < 0.0 ? -tiny : tiny;
    std::vector<double> x(m);
    unsigned st = seed * 2654435761u + 12345u;
    for (int i = 0; i < m; ++i) {
      st = st * 1664525u + 1013904223u;
      x[i] = static_cast<double>(st >> 8) / 16777216.0 - 0.5;
    }
    auto orth_normalize = [&] {
      for (int pass = 0; pass < 2; ++pass)
        for (const auto* v : against) {
          double dot = 0.0;
          for (int i = 0; i < m; ++i) dot += (*v)[i] * x[i];
          for (int i = 0; i < m; ++i) x[i] -= dot * (*v)[i];
        }
      double nrm = 0.0;
      for (double v : x) nrm += v * v;
      nrm = std::sqrt(nrm);
      if (nrm > 0.0)
        for (double& v : x) v /= nrm;
    };
    orth_normalize();
    for (int it = 0; it < 3; ++it) {
      // forward: the row operations of the factorization
      for (int i = 0; i + 1 < m; ++i) {
        if (piv[i]) std::swap(x[i], x[i + 1]);
        x[i + 1] -= l[i] * x[i];
      }
      // back substitution with the upper factor (two superdiagonals)
      for (int i = m - 1; i >= 0; --i) {
        double v = x[i];
        if (i + 1 < m) v -= u1[i] * x[i + 1];
        if (i + 2 < m) v -= u2[i] * x[i + 2];
        x[i] = v / u0[i];
      }
      double big = 0.0;
      for (double v : x) big = std::max(big, std::fabs(v));
      if (big > 0.0)
        for (double& v : x) v /= big;
      orth_normalize();
    }
    return x;
  }
};

// Reference selection order of Ritz values w (ascending) by `which`
// (lanczos_select_ritz_indices, src/core/RitzExtraction.cpp:162-179; sort_indices,
// include/fasteig_solver.hpp:58-82): sr, lr, sm, lm by a stable sort on the key, be
// alternating from the largest and the smallest.
inline std::vector<int32_t> ritz_order(const std::vector<double>& w, const std::string& which) {
  const int m = static_cast<int>(w.size());
  std::vector<int32_t> idx(m);
  for (int i = 0; i < m; ++i) idx[i] = i;
  if (which == "be") {
    int pos = 0;
    for (int i = 0; i < m / 2; ++i) {
      idx[pos++] = m - 1 - i;
      idx[pos++] = i;
    }
    if (m % 2 == 1) idx[pos] = m / 2;
    return idx;
  }
  auto key = [&](int i) {
    if (which == "sr") return w[i];
    if (which == "lr") return -w[i];
    if (which == "sm") return std::fabs(w[i]);
    return -std::fabs(w[i]);  // lm
  };
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return key(a) < key(b); });
  return idx;
}

// Eigenvalue indices (ascending order) that a selection of `nev` pairs by `which`
// (sr, lr, sm, lm, be) can draw from: both ends for lr/lm/be and sr, the window
// around zero for sm; all of them when the window covers the spectrum.
inline std::vector<int> tridiag_candidates(const TridiagEig& t, int nev, const char* which) {
  const int m = t.m;
  std::vector<int> idx;
  const std::string w(which);
  if (2 * nev >= m) {
    for (int i = 0; i < m; ++i) idx.push_back(i);
    return idx;
  }
  if (w == "sr") {
    for (int i = 0; i < nev; ++i) idx.push_back(i);
  } else if (w == "lr") {
    for (int i = m - nev; i < m; ++i) idx.push_back(i);
  } else if (w == "sm") {
    const int p = t.count_below(0.0);
    for (int i = std::max(0, p - nev); i < std::min(m, p + nev); ++i) idx.push_back(i);
  } else {  // lm, be: both ends
    for (int i = 0; i < nev; ++i) idx.push_back(i);
    for (int i = m - nev; i < m; ++i) idx.push_back(i);
  }
  return idx;
}

}  // namespace fe
