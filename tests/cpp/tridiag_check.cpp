// Driver for the host tridiagonal eigensolver (fasteig_b200/csrc/tridiag.hpp): reads
// m, then d[0..m), then e[0..m-1) from stdin; prints every eigenvalue in ascending
// order, then the eigenvectors (one per line), computed as the Lanczos snapshot does
// (inverse iteration, vectors of a cluster reorthogonalized).
#include <cstdio>
#include <vector>

#include "../../fasteig_b200/csrc/tridiag.hpp"

int main() {
  int m = 0;
  if (std::scanf("%d", &m) != 1 || m <= 0) return 2;
  std::vector<double> d(m), e(m > 1 ? m - 1 : 0);
  for (auto& v : d)
    if (std::scanf("%lf", &v) != 1) return 2;
  for (auto& v : e)
    if (std::scanf("%lf", &v) != 1) return 2;
  fe::TridiagEig t(d, e, m);
  std::vector<double> w(m);
  for (int j = 0; j < m; ++j) w[j] = t.eigenvalue(j);
  std::vector<std::vector<double>> vecs;
  for (int j = 0; j < m; ++j) {
    std::vector<const std::vector<double>*> cluster;
    for (int i = 0; i < j; ++i)
      if (std::fabs(w[i] - w[j]) <= 1e-3 * t.tnorm) cluster.push_back(&vecs[i]);
    vecs.push_back(t.vector(w[j], static_cast<unsigned>(j), cluster));
  }
  for (double v : w) std::printf("%.17g\n", v);
  for (const auto& x : vecs) {
    for (double v : x) std::printf("%.17g ", v);
    std::printf("\n");
  }
  // The snapshot's shortcut: selecting nev pairs among the candidate eigenvalues only
  // must give the selection over all of them. One line per (which, nev): 1 if equal.
  for (const char* which : {"sr", "lr", "sm", "lm", "be"}) {
    for (int nev : {1, 3, std::max(1, m / 3)}) {
      if (nev > m) continue;
      const std::vector<int32_t> full = fe::ritz_order(w, which);
      const std::vector<int> cand = fe::tridiag_candidates(t, nev, which);
      std::vector<double> cw;
      for (int c : cand) cw.push_back(t.eigenvalue(c));
      const std::vector<int32_t> part = fe::ritz_order(cw, which);
      bool same = true;
      for (int j = 0; j < nev; ++j) same = same && cw[part[j]] == w[full[j]];
      std::printf("select %s %d %d\n", which, nev, same ? 1 : 0);
    }
  }
  return 0;
}
