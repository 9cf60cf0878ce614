// Host-side minimum spanning tree for the per-cube clusterer's HDBSCAN
// backend (cluster/forward.py:103-128 runs the hdbscan package there).
//
// The cube's candidates are a few thousand points at most, so this is plain
// C++ on the host: O(n^2 d) arithmetic with O(n) memory, no device work.
//   D(a, b)   = sum over columns j (in order) of |X[a][j] - X[b][j]|  (float64)
//   core(a)   = the k-th smallest D(a, .) counting a itself as the 0-th,
//               k = clamp(min_samples, 1, n - 1)
//   M(a, b)   = max(D(a, b), core(a), core(b))      (mutual reachability)
// Prim's algorithm from point 0 over M: each step adds the outside point with
// the smallest distance to the tree (the first such index on a tie) and lowers
// the others' distances only when the new one is strictly smaller.  The
// edges come out in the order they were added: (source, point, distance).
#include "dsb_common.cuh"

#include <algorithm>
#include <cmath>
#include <limits>
#include <vector>

namespace {

inline double cityblock(const double* X, int d, int a, int b) {
  const double* xa = X + (size_t)a * d;
  const double* xb = X + (size_t)b * d;
  double s = 0.0;
  for (int j = 0; j < d; ++j) s += std::fabs(xa[j] - xb[j]);
  return s;
}

}  // namespace

extern "C" {

int dsb_cluster_mst(const double* X, int n, int d, int min_samples, double* core,
                    double* edges) {
  if (!X || !core || !edges || n < 2 || d <= 0 || min_samples < 0) return DSB_E_ARG;
  const int k = std::max(1, std::min(n - 1, min_samples));
  std::vector<double> row((size_t)n);
  for (int a = 0; a < n; ++a) {
    for (int b = 0; b < n; ++b) row[(size_t)b] = cityblock(X, d, a, b);
    std::nth_element(row.begin(), row.begin() + k, row.end());
    core[a] = row[(size_t)k];
  }
  std::vector<double> best((size_t)n);
  std::vector<int> src((size_t)n, 0);
  std::vector<char> in((size_t)n, 0);
  in[0] = 1;
  for (int b = 0; b < n; ++b)
    best[(size_t)b] = std::max(cityblock(X, d, 0, b), std::max(core[0], core[b]));
  for (int step = 0; step < n - 1; ++step) {
    int j = -1;
    double bj = std::numeric_limits<double>::infinity();
    for (int b = 0; b < n; ++b)
      if (!in[(size_t)b] && (j < 0 || best[(size_t)b] < bj)) {
        j = b;
        bj = best[(size_t)b];
      }
    edges[3 * (size_t)step] = src[(size_t)j];
    edges[3 * (size_t)step + 1] = j;
    edges[3 * (size_t)step + 2] = bj;
    in[(size_t)j] = 1;
    for (int b = 0; b < n; ++b) {
      if (in[(size_t)b]) continue;
      const double m = std::max(cityblock(X, d, j, b), std::max(core[j], core[b]));
      if (m < best[(size_t)b]) {
        best[(size_t)b] = m;
        src[(size_t)b] = j;
      }
    }
  }
  return DSB_OK;
}

}  // extern "C"
