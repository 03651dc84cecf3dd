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

// Nearest image of potential site `site` to the midpoint of the unit's
// segment, over the 27 lattice points around the rounded fractional
// coordinates; every lattice point outside that block is at least
// far_lattice away, which caps both bounds.  Bounds are shrunk by 1e-9
// relative and 1e-9 bohr and rounded down to float, so that they stay
// below the exact distances.
__device__ __forceinline__ SiteImage site_image(const DevSys &s,
                                                const DevWork &w, int unit,
                                                int site) {
  const DUnit u = w.units[unit];
  const DPair p = w.pairs[u.pair];
  double d[3], f[3];
#pragma unroll
  for (int x = 0; x < 3; ++x) {
    const double a = s.site_pos[3 * p.i + x];
    const double b = s.site_pos[3 * p.j + x] + p.L0[x] + s.cell[3 * u.cell + x];
    d[x] = 0.5 * (a + b) - s.psite_pos[3 * site + x];
  }
#pragma unroll
  for (int i = 0; i < 3; ++i)
    f[i] = rint(d[0] * s.inv[3 * i] + d[1] * s.inv[3 * i + 1] +
                d[2] * s.inv[3 * i + 2]);
  double b1 = 1e300, b2 = 1e300;
  int n1[3] = {0, 0, 0};
  for (int i = -1; i <= 1; ++i)
    for (int j = -1; j <= 1; ++j)
      for (int k = -1; k <= 1; ++k) {
        const double c0 = f[0] + i, c1 = f[1] + j, c2 = f[2] + k;
        double dd = 0.0;
#pragma unroll
        for (int x = 0; x < 3; ++x) {
          const double e = d[x] - (c0 * s.rv[x] + c1 * s.rv[3 + x] + c2 * s.rv[6 + x]);
          dd += e * e;
        }
        if (dd < b1) {
          b2 = b1;
          b1 = dd;
          n1[0] = (int)c0;
          n1[1] = (int)c1;
          n1[2] = (int)c2;
        } else if (dd < b2) {
          b2 = dd;
        }
      }
  SiteImage r;
  const bool fits = abs(n1[0]) < 32000 && abs(n1[1]) < 32000 && abs(n1[2]) < 32000;
  auto lower = [](double dist) {
    return __double2float_rd(fmax(0.0, dist * (1.0 - 1e-9) - 1e-9));
  };
  r.n[0] = fits ? (short)n1[0] : 0;
  r.n[1] = fits ? (short)n1[1] : 0;
  r.n[2] = fits ? (short)n1[2] : 0;
  r.pad = 0;
  // without a representable image both bounds are 0: the kernels then fall
  // back to the full search whenever the stored image is out of range
  r.d1 = fits ? lower(fmin(sqrt(b1), s.far_lattice)) : 0.f;
  r.d2 = fits ? lower(fmin(sqrt(b2), s.far_lattice)) : 0.f;
  return r;
}

// True when a point at least d - pm from every lattice point of interest
// is certainly outside the screening radius^2 t: the float lower bound of
// d - pm (pmf >= pm, rounded down) squared, rounded down, exceeds tf >= t.
__device__ __forceinline__ bool beyond(float d, float pmf, float tf) {
  const float a = __fsub_rd(d, pmf);
  return a > 0.f && __fmul_rd(a, a) > tf;
}

// Closest-image search of a three-centre screen (the findLatticeVector step
// of nuclearPE/electronicPE, integrals.F90:2632,2791) for the point Ps with
// |Ps - M| = pm, radius^2 t.  Returns false when no image of site C lies
// within the radius; otherwise sets L2, the lattice vector from which the
// images in range are enumerated, and v = Ps - C - L2 with |v|^2 <= t.  With
// the stored midpoint image: no lattice point is nearer to Ps - C than
// d1 - pm, none but the stored one nearer than d2 - pm.  pmf and tf are
// float upper bounds of pm and t for those tests.
__device__ __forceinline__ bool site_search(const DevSys &s, const DevWork &w,
                                            int unit, int site,
                                            const double Ps[3], float pmf,
                                            double t, float tf, double L2[3],
                                            double v[3], double &c0) {
  const double *C = s.psite_pos + 3 * site;
  if (w.simg) {
    const SiteImage im = w.simg[(long long)unit * s.nps + site];
    if (beyond(im.d1, pmf, tf)) return false;
    double c = 0.0;
#pragma unroll
    for (int x = 0; x < 3; ++x) {
      L2[x] = im.n[0] * s.rv[x] + im.n[1] * s.rv[3 + x] + im.n[2] * s.rv[6 + x];
      v[x] = Ps[x] - C[x] - L2[x];
      c += v[x] * v[x];
    }
    if (c <= t) {
      c0 = c;
      return true;
    }
    if (beyond(im.d2, pmf, tf)) return false;
  }
  double d[3];
#pragma unroll
  for (int x = 0; x < 3; ++x) d[x] = Ps[x] - C[x];
  nearest_lattice(s, d, L2);
  c0 = 0.0;
#pragma unroll
  for (int x = 0; x < 3; ++x) {
    v[x] = Ps[x] - C[x] - L2[x];
    c0 += v[x] * v[x];
  }
  return c0 <= t;
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
