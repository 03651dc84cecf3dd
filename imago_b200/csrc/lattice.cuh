// lattice.cuh -- lattice point lists of the reference's initializeLattice
// (lattice.f90:310-782), shared by the integral set-up and the SCF set-up.
#pragma once

#include <cmath>
#include <numeric>
#include <utility>
#include <vector>

namespace imago {

// cellBorderCheck (lattice.f90:698-782): a lattice point beyond the limit
// is kept when one of the seven other corners of the cell it spans, walked
// in the reference's order, lies within it.
inline bool lattice_border_within(const double *rv, const double *t, double lim) {
  double sh[3] = {0, 0, 0}, cur[3] = {t[0], t[1], t[2]};
  for (int i = 0; i < 3; ++i)
    for (int x = 0; x < 3; ++x) sh[x] += rv[3 * i + x];
  const int ax[7] = {0, 1, 0, 2, 0, 1, 0};
  const int sg[7] = {1, 1, -1, 1, 1, -1, -1};
  for (int s = 0; s < 7; ++s) {
    cur[ax[s]] += sg[s] * sh[ax[s]];
    if (cur[0] * cur[0] + cur[1] * cur[1] + cur[2] * cur[2] < lim) return true;
  }
  return false;
}

// The order makeLattice's mergeSort (sortSubs.f90:18-200) leaves: runs of
// one merged pairwise, bottom up, the last odd run carried; a head of the
// first run goes first only when strictly smaller, so among equal keys the
// later run's element leads.  (The cells of one |R|^2 shell come out in
// this order in the reference; a stable sort would keep loop order.)
template <class T, class Less>
void merge_runs_like_reference(std::vector<T> &v, Less less) {
  const size_t n = v.size();
  if (n < 2) return;
  std::vector<T> other(n);
  std::vector<size_t> edge(n + 1);
  std::iota(edge.begin(), edge.end(), size_t(0));
  std::vector<T> *src = &v, *dst = &other;
  size_t runs = n;
  while (runs > 1) {
    size_t out = 0;
    for (size_t r = 0; r < runs / 2; ++r) {
      size_t a = edge[2 * r], a_end = edge[2 * r + 1], b = a_end, b_end = edge[2 * r + 2];
      while (a < a_end && b < b_end)
        (*dst)[out++] = less((*src)[a], (*src)[b]) ? (*src)[a++] : (*src)[b++];
      while (a < a_end) (*dst)[out++] = (*src)[a++];
      while (b < b_end) (*dst)[out++] = (*src)[b++];
      edge[r + 1] = b_end;
    }
    if (runs % 2) {
      for (size_t i = out; i < edge[runs]; ++i) (*dst)[i] = (*src)[i];
      edge[runs / 2 + 1] = edge[runs];
    }
    runs = runs / 2 + runs % 2;
    std::swap(src, dst);
  }
  if (src != &v) v.swap(*src);
}


// getNumCells + makeLattice (lattice.f90:469-696): the points n0 a + n1 b +
// n2 c of the lattice spanned by vectors[3 * abc + xyz], n_i in
// [-(reps_i - 1) / 2, reps_i / 2] with reps_i = 2 ceil(sqrt(lim) / |v_i|) + 1,
// within |R|^2 <= lim or kept by the border check, ordered by |R|^2 as the
// reference's merge sort leaves them.  dims [n][3], sizes [n] = |R|^2.
inline void lattice_points(const double *vectors, double lim, std::vector<double> &dims,
                           std::vector<double> &sizes) {
  int reps[3];
  for (int i = 0; i < 3; ++i) {
    double len2 = 0.0;
    for (int x = 0; x < 3; ++x) len2 += vectors[3 * i + x] * vectors[3 * i + x];
    reps[i] = 2 * (int)std::ceil(std::sqrt(lim) / std::sqrt(len2)) + 1;
  }
  struct Point {
    double size, d[3];
  };
  std::vector<Point> list;
  for (int i = 1; i <= reps[0]; ++i)
    for (int j = 1; j <= reps[1]; ++j)
      for (int k = 1; k <= reps[2]; ++k) {
        const int rep[3] = {i - (1 + reps[0]) / 2, j - (1 + reps[1]) / 2,
                            k - (1 + reps[2]) / 2};
        double t[3] = {0, 0, 0};
        for (int l = 0; l < 3; ++l)
          for (int m = 0; m < 3; ++m) t[m] = t[m] + vectors[3 * l + m] * rep[l];
        const double s = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
        if (s > lim && !lattice_border_within(vectors, t, lim)) continue;
        list.push_back({s, {t[0], t[1], t[2]}});
      }
  merge_runs_like_reference(list, [](const Point &a, const Point &b) { return a.size < b.size; });
  dims.resize(3 * list.size());
  sizes.resize(list.size());
  for (size_t i = 0; i < list.size(); ++i) {
    for (int x = 0; x < 3; ++x) dims[3 * i + x] = list[i].d[x];
    sizes[i] = list[i].size;
  }
}

}  // namespace imago
