// geom.cuh -- per-shell-pair geometry shared by the primitive kernels.
#pragma once

#include "intg.cuh"

namespace imago {

// Nearest lattice vector to v: round the fractional coordinates, then take
// the closest of that lattice point and its 26 neighbours.  This is the
// role of findLatticeVector (lattice.f90:784-888).
__device__ __forceinline__ void nearest_lattice(const DevSys &s,
                                                const double v[3],
                                                double out[3]) {
  double base[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const double f = v[0] * s.inv[3 * i] + v[1] * s.inv[3 * i + 1] +
                     v[2] * s.inv[3 * i + 2];
    double r = (double)(long long)(fabs(f) + 0.5);
    if (f < 0.0) r = -r;
#pragma unroll
    for (int x = 0; x < 3; ++x) base[x] += s.rv[3 * i + x] * r;
  }
  double best[3] = {base[0], base[1], base[2]};
  double bd = 0.0;
#pragma unroll
  for (int x = 0; x < 3; ++x) bd += (v[x] - base[x]) * (v[x] - base[x]);
  for (int i = -1; i <= 1; ++i)
    for (int j = -1; j <= 1; ++j)
      for (int k = -1; k <= 1; ++k) {
        if (!i && !j && !k) continue;
        double cand[3], d = 0.0;
#pragma unroll
        for (int x = 0; x < 3; ++x) {
          cand[x] = base[x] + i * s.rv[x] + j * s.rv[3 + x] + k * s.rv[6 + x];
          d += (v[x] - cand[x]) * (v[x] - cand[x]);
        }
        if (d < bd * (1.0 - 1e-12)) {
          bd = d;
          best[0] = cand[0];
          best[1] = cand[1];
          best[2] = cand[2];
        }
      }
  out[0] = best[0];
  out[1] = best[1];
  out[2] = best[2];
}

struct SpGeom {
  double A[3], B[3];   // atom 1, shifted atom 2
  double a1, a2;       // primitive exponents
  double a1s, a2s;     // exponents of the element's first type (screening)
  double r2;
  int ti, tj;
};

__device__ __forceinline__ SpGeom sp_geom(const DevSys &s, const DevWork &w,
                                          const DSp &sp) {
  SpGeom g;
  const DUnit u = w.units[sp.unit];
  const DPair p = w.pairs[u.pair];
#pragma unroll
  for (int x = 0; x < 3; ++x) {
    g.A[x] = s.site_pos[3 * p.i + x];
    g.B[x] = s.site_pos[3 * p.j + x] + p.L0[x] + s.cell[3 * u.cell + x];
  }
  g.ti = p.ti;
  g.tj = p.tj;
  g.a1 = s.alpha[s.type_alpha_off[p.ti] + sp.a];
  g.a2 = s.alpha[s.type_alpha_off[p.tj] + sp.b];
  g.a1s = s.alpha[s.type_alpha_off[s.type_screen[p.ti]] + sp.a];
  g.a2s = s.alpha[s.type_alpha_off[s.type_screen[p.tj]] + sp.b];
  g.r2 = u.r2;
  return g;
}

}  // namespace imago
