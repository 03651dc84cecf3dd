// k_prim.cu -- primitive shell-pair blocks per class.
//
// Shell pairs are sorted by class; each s/p/d class runs a fully unrolled
// kernel, the f classes share runtime-class kernels.
#include <algorithm>

#include "geom.cuh"
#include "prim.cuh"

namespace imago {

// ------------------------------------------------------------ prim2c --
template <int LA, int LB, bool KIN>
__global__ void __launch_bounds__(128)
    k_prim2c(DevSys s, DevWork w, int beg, int end, double *blk) {
  const int g = beg + blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= end) return;
  const DSp sp = w.sps[w.sp_by_cls[g]];
  const SpGeom q = sp_geom(s, w, sp);
  prim2c<LA, LB, KIN>(q.a1, q.a2, q.A, q.B, blk + sp.boff);
}

// Mass velocity (built once per SCF run, rel = 1): s/p/d classes unrolled,
// the f classes through one runtime-class kernel.
template <int LA, int LB>
__global__ void __launch_bounds__(128)
    k_prim_mv(DevSys s, DevWork w, int beg, int end, double *blk) {
  const int g = beg + blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= end) return;
  const DSp sp = w.sps[w.sp_by_cls[g]];
  const SpGeom q = sp_geom(s, w, sp);
  prim_mv<LA, LB>(q.a1, q.a2, q.A, q.B, -kMassVelPref, blk + sp.boff);
}

__global__ void __launch_bounds__(128)
    k_prim_mv_rt(DevSys s, DevWork w, int beg, int end, int la, int lb,
                 double *blk) {
  const int g = beg + blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= end) return;
  const DSp sp = w.sps[w.sp_by_cls[g]];
  const SpGeom q = sp_geom(s, w, sp);
  prim_mv_rt(la, lb, q.a1, q.a2, q.A, q.B, -kMassVelPref, blk + sp.boff);
}

// Momentum / dipole: three component blocks per shell pair, component c at
// blk + c * blk_total.
template <int LA, int LB, bool DIP>
__global__ void __launch_bounds__(128)
    k_prim_vec(DevSys s, DevWork w, int beg, int end, double3 center, double *blk) {
  const int g = beg + blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= end) return;
  const DSp sp = w.sps[w.sp_by_cls[g]];
  const SpGeom q = sp_geom(s, w, sp);
  const double C[3] = {center.x, center.y, center.z};
  prim_vec<LA, LB, DIP>(q.a1, q.a2, q.A, q.B, C, blk + sp.boff, w.blk_total);
}

template <bool DIP>
__global__ void __launch_bounds__(128)
    k_prim_vec_rt(DevSys s, DevWork w, int beg, int end, int la, int lb,
                  double3 center, double *blk) {
  const int g = beg + blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= end) return;
  const DSp sp = w.sps[w.sp_by_cls[g]];
  const SpGeom q = sp_geom(s, w, sp);
  const double C[3] = {center.x, center.y, center.z};
  prim_vec_rt<DIP>(la, lb, q.a1, q.a2, q.A, q.B, C, blk + sp.boff, w.blk_total);
}

// ------------------------------------------------------------ prim3c --
// One thread per (shell pair, term).  The site and lattice-image loops are
// those of nuclearPE (integrals.F90:2533-2698) and electronicPE
// (2700-2858): a closest-image screen per site, then the images of that
// site within threeAlphaDist of the overlap centre, in |R| order.
// Registers: four CTAs per SM up to d-p (a few bytes of spill for d-p),
// three for d-d, whose Hermite accumulator alone holds 35 doubles.
// One item g < n * nterm of class (LA, LB): term g / n, shell pair g % n of
// the class's list.  Shared by the per-class launches and the work queue.
// CNT: the same loops, counting the screened (site, image) triples into
// *ntrip instead of integrating (nothing is written).
template <int LA, int LB, bool NUC, bool CNT = false>
__device__ __forceinline__ void prim3c_item(const DevSys &s, const DevWork &w, int beg,
                                            int n, const Term3c *terms, double *blk,
                                            long long g, unsigned *ntrip = nullptr) {
  constexpr int L = LA + LB;
  const int tl = (int)(g / n);
  const DSp sp = w.sps[w.sp_by_cls[beg + (int)(g % n)]];
  const SpGeom q = sp_geom(s, w, sp);
  const Term3c tm = terms[tl];

  // alphaDist / alphaCenter (gaussRelations.f90:112-131) from the element's
  // first-type exponents, as the reference tables are built.
  const double cen = q.a1s / (q.a1s + q.a2s);
  const double adist = s.T / q.a2s / cen;
  const double frac = 1 - q.r2 / adist;
  double Ps[3], Pt[3];
  const double zeta = q.a1 + q.a2, xi = q.a1 * q.a2 / zeta;
  double pm = 0.0;  // |Ps - M|, M the midpoint of A and B
#pragma unroll
  for (int x = 0; x < 3; ++x) {
    Ps[x] = cen * (q.A[x] - q.B[x]) + q.B[x];
    Pt[x] = (q.a1 * q.A[x] + q.a2 * q.B[x]) / zeta;
    const double e = Ps[x] - 0.5 * (q.A[x] + q.B[x]);
    pm += e * e;
  }
  pm = sqrt(pm);
  double Q[nherm(L)];
#pragma unroll
  for (int i = 0; i < nherm(L); ++i) Q[i] = 0.0;

  // NP runs over every potential type, EP over the term's type; sites of a
  // type are contiguous and types come in site order.
  const int pt0 = NUC ? 0 : tm.ptype, pt1 = NUC ? s.npt : tm.ptype + 1;
  double tcut = 0.0, a3 = 0.0;
  if (!NUC) {
    const int pt = tm.ptype;
    a3 = s.palpha[s.ptype_alpha_off[pt] + tm.j];
    const double a3s = s.palpha[s.ptype_alpha_off[s.ptype_screen[pt]] + tm.j];
    // alphaPotDist (gaussRelations.f90:187-196)
    tcut = frac * (s.T * (q.a1s + q.a2s + a3s) / (q.a1s + q.a2s) / a3s);
  }
  const double z3e = zeta + a3, mue = zeta * a3 / z3e;
  const float pmf = __double2float_ru(pm);

  for (int pt = pt0; pt < pt1; ++pt) {
    double w0 = 1.0, mu = mue, nu = 0.0, t = tcut;
    if (NUC) {
      const double Z = s.ptype_z[pt];
      if (Z < kSmallThresh) continue;
      const double an = s.ptype_nucalpha[pt];
      const double ans = s.ptype_nucalpha[s.ptype_screen[pt]];
      // alphaNucDist (gaussRelations.f90:262-270)
      t = frac * (s.T * (q.a1s + q.a2s + ans) / (q.a1s + q.a2s) / ans);
      const double z3 = zeta + an;
      mu = zeta * an / z3;
      nu = zeta * zeta / z3;
      w0 = -Z * (2.0 * kPi / z3);
    }
    const float tf = __double2float_ru(t);
    const int s0 = s.ptype_first_site[pt], s1 = s0 + s.ptype_mult[pt];
    // the type's sites nearest the unit first (with the site tables): the
    // first one beyond reach ends the walk; without them, every site
    const long long ub = (long long)sp.unit * s.nps;
    for (int r = 0; r < s1 - s0; ++r) {
      int site = s0 + r;
      if (w.site_rank) {
        site = s0 + w.site_rank[ub + s0 + r];
        if (beyond(w.simg[ub + site].d1, pmf, tf)) break;
      }
      double L2[3], v[3], c0;
      if (!site_search(s, w, sp.unit, site, Ps, pmf, t, tf, L2, v, c0)) continue;
      const double *C = s.psite_pos + 3 * site;
      const double maxr = c0 + t + 2.0 * sqrt(c0 * t);
      for (int nc = 0; nc < s.ncell; ++nc) {
        if (s.csize[nc] > maxr) break;
        const double *R = s.cell + 3 * nc;
        const double dx = v[0] - R[0], dy = v[1] - R[1], dz = v[2] - R[2];
        if (dx * dx + dy * dy + dz * dz > t) continue;
        if constexpr (CNT) {
          ++*ntrip;
        } else {
          double X[3];
#pragma unroll
          for (int x = 0; x < 3; ++x) X[x] = Pt[x] - (C[x] + L2[x] + R[x]);
          if (NUC)
            accumulate_nuclear_q<L>(X, mu, nu, w0, Q);
          else
            accumulate_overlap_q<L>(X, mu, 1.0, Q);
        }
      }
    }
  }
  if constexpr (!CNT) {
    const double pref = NUC ? exp(-xi * q.r2) : pow(kPi / z3e, 1.5) * exp(-xi * q.r2);
    hermite_to_sh<LA, LB>(q.A, q.B, q.a1, q.a2, pref, Q,
                          blk + (long long)tl * w.blk_total + sp.boff);
  }
}

// The Hermite-to-spherical transform of one term of a pair, as a call: the
// other term's accumulators wait in memory meanwhile instead of crowding
// the transform's registers.
template <int LA, int LB>
__device__ __noinline__ void pair_to_sh(const double *A, const double *B, double a1, double a2,
                                        double pref, const double *Q, double *out) {
  double Qr[nherm(LA + LB)];
#pragma unroll
  for (int i = 0; i < nherm(LA + LB); ++i) Qr[i] = Q[i];
  hermite_to_sh<LA, LB>(A, B, a1, a2, pref, Qr, out);
}

// Two EP terms of one potential type per thread (group g / n of tg): the
// sites and images are walked once with the larger of the two screening
// radii and each image is accumulated into the terms whose own radius it
// passes, so each term gets exactly the triples of its own walk (the set
// of images within a radius does not depend on the lattice vector the
// enumeration starts from).
template <int LA, int LB>
__device__ __forceinline__ void prim3c_item2(const DevSys &s, const DevWork &w, int beg,
                                             int n, const Term3c *terms,
                                             const TermGroups &tg, double *blk, long long g) {
  constexpr int L = LA + LB;
  const int gi = (int)(g / n);
  const int t0 = tg.first[gi], cnt = tg.count[gi];
  const DSp sp = w.sps[w.sp_by_cls[beg + (int)(g % n)]];
  const SpGeom q = sp_geom(s, w, sp);
  const double cen = q.a1s / (q.a1s + q.a2s);
  const double adist = s.T / q.a2s / cen;
  const double frac = 1 - q.r2 / adist;
  double Ps[3], Pt[3];
  const double zeta = q.a1 + q.a2, xi = q.a1 * q.a2 / zeta;
  double pm = 0.0;
#pragma unroll
  for (int x = 0; x < 3; ++x) {
    Ps[x] = cen * (q.A[x] - q.B[x]) + q.B[x];
    Pt[x] = (q.a1 * q.A[x] + q.a2 * q.B[x]) / zeta;
    const double e = Ps[x] - 0.5 * (q.A[x] + q.B[x]);
    pm += e * e;
  }
  pm = sqrt(pm);
  const int pt = terms[t0].ptype;
  double tc[2], mu[2], a3[2];
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const Term3c tm = terms[t0 + (j < cnt ? j : 0)];
    a3[j] = s.palpha[s.ptype_alpha_off[pt] + tm.j];
    const double a3s = s.palpha[s.ptype_alpha_off[s.ptype_screen[pt]] + tm.j];
    // alphaPotDist (gaussRelations.f90:187-196); a missing second term
    // takes no image
    tc[j] = j < cnt ? frac * (s.T * (q.a1s + q.a2s + a3s) / (q.a1s + q.a2s) / a3s) : -1.0;
    mu[j] = zeta * a3[j] / (zeta + a3[j]);
  }
  const double t = fmax(tc[0], tc[1]);
  const float tf = __double2float_ru(t), pmf = __double2float_ru(pm);
  double Q[2][nherm(L)];
#pragma unroll
  for (int j = 0; j < 2; ++j)
#pragma unroll
    for (int i = 0; i < nherm(L); ++i) Q[j][i] = 0.0;
  const int s0 = s.ptype_first_site[pt], s1 = s0 + s.ptype_mult[pt];
  const long long ub = (long long)sp.unit * s.nps;
  for (int r = 0; r < s1 - s0; ++r) {
    int site = s0 + r;
    if (w.site_rank) {
      site = s0 + w.site_rank[ub + s0 + r];
      if (beyond(w.simg[ub + site].d1, pmf, tf)) break;
    }
    double L2[3], v[3], c0;
    if (!site_search(s, w, sp.unit, site, Ps, pmf, t, tf, L2, v, c0)) continue;
    const double *C = s.psite_pos + 3 * site;
    const double maxr = c0 + t + 2.0 * sqrt(c0 * t);
    for (int nc = 0; nc < s.ncell; ++nc) {
      if (s.csize[nc] > maxr) break;
      const double *R = s.cell + 3 * nc;
      const double dx = v[0] - R[0], dy = v[1] - R[1], dz = v[2] - R[2];
      const double d2 = dx * dx + dy * dy + dz * dz;
      if (d2 > t) continue;
      double X[3];
#pragma unroll
      for (int x = 0; x < 3; ++x) X[x] = Pt[x] - (C[x] + L2[x] + R[x]);
      if (d2 <= tc[0]) accumulate_overlap_q<L>(X, mu[0], 1.0, Q[0]);
      if (d2 <= tc[1]) accumulate_overlap_q<L>(X, mu[1], 1.0, Q[1]);
    }
  }
  const double ex = exp(-xi * q.r2);
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    if (j >= cnt) break;
    const double pref = pow(kPi / (zeta + a3[j]), 1.5) * ex;
    pair_to_sh<LA, LB>(q.A, q.B, q.a1, q.a2, pref, Q[j],
                       blk + (long long)(t0 + j) * w.blk_total + sp.boff);
  }
}

template <int LA, int LB>
__global__ void __launch_bounds__(128, LA + LB >= 3 ? 3 : 4)
    k_prim3c_pair(DevSys s, DevWork w, int beg, int n, const Term3c *terms, TermGroups tg,
                  double *blk) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= (long long)n * tg.n) return;
  prim3c_item2<LA, LB>(s, w, beg, n, terms, tg, blk, g);
}

// Screened primitive triples (shell pair, potential site, lattice image) of
// one class's items: what the reference's nuclearPE / electronicPE loops
// evaluate (integrals.F90:2533-2698, 2700-2858), summed into *count.
template <int LA, int LB, bool NUC>
__global__ void __launch_bounds__(128)
    k_prim3c_count(DevSys s, DevWork w, int beg, int n, const Term3c *terms, int nterm,
                   unsigned long long *count) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned c = 0;
  if (g < (long long)n * nterm)
    prim3c_item<LA, LB, NUC, true>(s, w, beg, n, terms, nullptr, g, &c);
  c = __reduce_add_sync(0xffffffffu, c);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, (unsigned long long)c);
}

template <int LA, int LB, bool NUC>
__global__ void __launch_bounds__(128, LA + LB >= 4 ? 3 : (LA + LB >= 3 ? 4 : (LA + LB == 2 ? 5 : 6)))
    k_prim3c(DevSys s, DevWork w, int beg, int n, const Term3c *terms,
             int nterm, double *blk) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= (long long)n * nterm) return;
  prim3c_item<LA, LB, NUC>(s, w, beg, n, terms, blk, g);
}

// The potential terms of the PSCF Hamiltonian (gaussOverlapHamPSCF,
// integrals.F90:3240-3442) for one spin, fused: T adjacent lanes of a warp
// share a shell pair, each running the site and image loops of k_prim3c for
// every T-th term, weighting the term by its coefficient coef[t] times
// (pi/z3)^1.5, into its Hermite accumulator; the T accumulators are summed
// by warp shuffles and the first lane writes one Hermite-to-spherical
// transform to H + sp.boff.  The per-term blocks of the EP build are never
// formed.  T > 1 gives a small system's shell pairs enough threads.
template <int LA, int LB, int T>
__global__ void __launch_bounds__(128, LA + LB >= 4 ? 3 : 4)
    k_prim3c_ham(DevSys s, DevWork w, int beg, int n, const Term3c *terms, int nterm,
                 const double *coef, double *H) {
  constexpr int L = LA + LB;
  static_assert(32 % T == 0, "a shell pair's lanes stay in one warp");
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int pair = (int)(g / T), sub = (int)(g % T);
  // lanes past the last pair stay for the shuffles below
  const bool live = pair < n;
  double Q[nherm(L)];
#pragma unroll
  for (int i = 0; i < nherm(L); ++i) Q[i] = 0.0;
  DSp sp{};
  SpGeom q{};
  if (live) {
    sp = w.sps[w.sp_by_cls[beg + pair]];
    q = sp_geom(s, w, sp);
    const double cen = q.a1s / (q.a1s + q.a2s);
    const double adist = s.T / q.a2s / cen;
    const double frac = 1 - q.r2 / adist;
    double Ps[3], Pt[3];
    const double zeta = q.a1 + q.a2;
    double pm = 0.0;
#pragma unroll
    for (int x = 0; x < 3; ++x) {
      Ps[x] = cen * (q.A[x] - q.B[x]) + q.B[x];
      Pt[x] = (q.a1 * q.A[x] + q.a2 * q.B[x]) / zeta;
      const double e = Ps[x] - 0.5 * (q.A[x] + q.B[x]);
      pm += e * e;
    }
    pm = sqrt(pm);
    const float pmf = __double2float_ru(pm);
    for (int tl = sub; tl < nterm; tl += T) {
      const Term3c tm = terms[tl];
      const int pt = tm.ptype;
      const double a3 = s.palpha[s.ptype_alpha_off[pt] + tm.j];
      const double a3s = s.palpha[s.ptype_alpha_off[s.ptype_screen[pt]] + tm.j];
      // alphaPotDist (gaussRelations.f90:187-196)
      const double t = frac * (s.T * (q.a1s + q.a2s + a3s) / (q.a1s + q.a2s) / a3s);
      const double z3e = zeta + a3, mu = zeta * a3 / z3e;
      const double wt = coef[tl] * pow(kPi / z3e, 1.5);
      const float tf = __double2float_ru(t);
      const int s0 = s.ptype_first_site[pt], s1 = s0 + s.ptype_mult[pt];
      for (int cb = s0 - s0 % kSiteCluster; cb < s1; cb += kSiteCluster) {
        if (w.cl_d1 &&
            beyond(w.cl_d1[(long long)sp.unit * w.ncl + cb / kSiteCluster], pmf, tf))
          continue;
        const int lo = max(cb, s0), hi = min(cb + kSiteCluster, s1);
        for (int site = lo; site < hi; ++site) {
          double L2[3], v[3], c0;
          if (!site_search(s, w, sp.unit, site, Ps, pmf, t, tf, L2, v, c0)) continue;
          const double *C = s.psite_pos + 3 * site;
          const double maxr = c0 + t + 2.0 * sqrt(c0 * t);
          for (int nc = 0; nc < s.ncell; ++nc) {
            if (s.csize[nc] > maxr) break;
            const double *R = s.cell + 3 * nc;
            const double dx = v[0] - R[0], dy = v[1] - R[1], dz = v[2] - R[2];
            if (dx * dx + dy * dy + dz * dz > t) continue;
            double X[3];
#pragma unroll
            for (int x = 0; x < 3; ++x) X[x] = Pt[x] - (C[x] + L2[x] + R[x]);
            accumulate_overlap_q<L>(X, mu, wt, Q);
          }
        }
      }
    }
  }
  if (T > 1) {
#pragma unroll
    for (int off = T / 2; off > 0; off /= 2)
#pragma unroll
      for (int i = 0; i < nherm(L); ++i) Q[i] += __shfl_xor_sync(0xffffffffu, Q[i], off);
  }
  if (!live || sub != 0) return;
  const double xi = q.a1 * q.a2 / (q.a1 + q.a2);
  hermite_to_sh<LA, LB>(q.A, q.B, q.a1, q.a2, exp(-xi * q.r2), Q, H + sp.boff);
}

// f classes of k_prim3c_ham, runtime loops.
__global__ void __launch_bounds__(128)
    k_prim3c_ham_rt(DevSys s, DevWork w, int beg, int n, const Term3c *terms,
                    int nterm, const double *coef, int la, int lb, double *H) {
  const int L = la + lb;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  const DSp sp = w.sps[w.sp_by_cls[beg + g]];
  const SpGeom q = sp_geom(s, w, sp);
  const double cen = q.a1s / (q.a1s + q.a2s);
  const double adist = s.T / q.a2s / cen;
  const double frac = 1 - q.r2 / adist;
  double Ps[3], Pt[3];
  const double zeta = q.a1 + q.a2, xi = q.a1 * q.a2 / zeta;
  double pm = 0.0;
  for (int x = 0; x < 3; ++x) {
    Ps[x] = cen * (q.A[x] - q.B[x]) + q.B[x];
    Pt[x] = (q.a1 * q.A[x] + q.a2 * q.B[x]) / zeta;
    const double e = Ps[x] - 0.5 * (q.A[x] + q.B[x]);
    pm += e * e;
  }
  pm = sqrt(pm);
  const float pmf = __double2float_ru(pm);
  double Q[kMaxHerm];
  for (int i = 0; i < kMaxHerm; ++i) Q[i] = 0.0;
  for (int tl = 0; tl < nterm; ++tl) {
    const Term3c tm = terms[tl];
    const int pt = tm.ptype;
    const double a3 = s.palpha[s.ptype_alpha_off[pt] + tm.j];
    const double a3s = s.palpha[s.ptype_alpha_off[s.ptype_screen[pt]] + tm.j];
    const double t = frac * (s.T * (q.a1s + q.a2s + a3s) / (q.a1s + q.a2s) / a3s);
    const double z3e = zeta + a3, mu = zeta * a3 / z3e;
    const double wt = coef[tl] * pow(kPi / z3e, 1.5);
    const float tf = __double2float_ru(t);
    const int s0 = s.ptype_first_site[pt], s1 = s0 + s.ptype_mult[pt];
    for (int cb = s0 - s0 % kSiteCluster; cb < s1; cb += kSiteCluster) {
      if (w.cl_d1 &&
          beyond(w.cl_d1[(long long)sp.unit * w.ncl + cb / kSiteCluster], pmf, tf))
        continue;
      const int lo = max(cb, s0), hi = min(cb + kSiteCluster, s1);
      for (int site = lo; site < hi; ++site) {
        double L2[3], v[3], c0;
        if (!site_search(s, w, sp.unit, site, Ps, pmf, t, tf, L2, v, c0)) continue;
        const double *C = s.psite_pos + 3 * site;
        const double maxr = c0 + t + 2.0 * sqrt(c0 * t);
        for (int nc = 0; nc < s.ncell; ++nc) {
          if (s.csize[nc] > maxr) break;
          const double *R = s.cell + 3 * nc;
          const double dx = v[0] - R[0], dy = v[1] - R[1], dz = v[2] - R[2];
          if (dx * dx + dy * dy + dz * dz > t) continue;
          double X[3];
          for (int x = 0; x < 3; ++x) X[x] = Pt[x] - (C[x] + L2[x] + R[x]);
          accumulate_overlap_q_rt(L, X, mu, wt, Q);
        }
      }
    }
  }
  hermite_to_sh_rt(la, lb, q.A, q.B, q.a1, q.a2, exp(-xi * q.r2), Q, H + sp.boff);
}

// f classes: one runtime-class kernel each for 2C and 3C.
template <bool KIN>
__global__ void __launch_bounds__(128)
    k_prim2c_rt(DevSys s, DevWork w, int beg, int end, int la, int lb,
                double *blk) {
  const int g = beg + blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= end) return;
  const DSp sp = w.sps[w.sp_by_cls[g]];
  const SpGeom q = sp_geom(s, w, sp);
  prim2c_rt(la, lb, KIN, q.a1, q.a2, q.A, q.B, blk + sp.boff);
}

template <bool NUC>
__device__ __noinline__ void prim3c_item_rt(const DevSys &s, const DevWork &w, int beg,
                                            int n, const Term3c *terms, int la, int lb,
                                            double *blk, long long g) {
  const int L = la + lb;
  const int tl = (int)(g / n);
  const DSp sp = w.sps[w.sp_by_cls[beg + (int)(g % n)]];
  const SpGeom q = sp_geom(s, w, sp);
  const Term3c tm = terms[tl];
  const double cen = q.a1s / (q.a1s + q.a2s);
  const double adist = s.T / q.a2s / cen;
  const double frac = 1 - q.r2 / adist;
  double Ps[3], Pt[3];
  const double zeta = q.a1 + q.a2, xi = q.a1 * q.a2 / zeta;
  double pm = 0.0;  // |Ps - M|, M the midpoint of A and B
  for (int x = 0; x < 3; ++x) {
    Ps[x] = cen * (q.A[x] - q.B[x]) + q.B[x];
    Pt[x] = (q.a1 * q.A[x] + q.a2 * q.B[x]) / zeta;
    const double e = Ps[x] - 0.5 * (q.A[x] + q.B[x]);
    pm += e * e;
  }
  pm = sqrt(pm);
  double Q[kMaxHerm];
  for (int i = 0; i < kMaxHerm; ++i) Q[i] = 0.0;
  // NP runs over every potential type, EP over the term's type; sites of a
  // type are contiguous and types come in site order.
  const int pt0 = NUC ? 0 : tm.ptype, pt1 = NUC ? s.npt : tm.ptype + 1;
  double tcut = 0.0, a3 = 0.0;
  if (!NUC) {
    const int pt = tm.ptype;
    a3 = s.palpha[s.ptype_alpha_off[pt] + tm.j];
    const double a3s = s.palpha[s.ptype_alpha_off[s.ptype_screen[pt]] + tm.j];
    // alphaPotDist (gaussRelations.f90:187-196)
    tcut = frac * (s.T * (q.a1s + q.a2s + a3s) / (q.a1s + q.a2s) / a3s);
  }
  const double z3e = zeta + a3, mue = zeta * a3 / z3e;
  const float pmf = __double2float_ru(pm);

  for (int pt = pt0; pt < pt1; ++pt) {
    double w0 = 1.0, mu = mue, nu = 0.0, t = tcut;
    if (NUC) {
      const double Z = s.ptype_z[pt];
      if (Z < kSmallThresh) continue;
      const double an = s.ptype_nucalpha[pt];
      const double ans = s.ptype_nucalpha[s.ptype_screen[pt]];
      // alphaNucDist (gaussRelations.f90:262-270)
      t = frac * (s.T * (q.a1s + q.a2s + ans) / (q.a1s + q.a2s) / ans);
      const double z3 = zeta + an;
      mu = zeta * an / z3;
      nu = zeta * zeta / z3;
      w0 = -Z * (2.0 * kPi / z3);
    }
    const float tf = __double2float_ru(t);
    const int s0 = s.ptype_first_site[pt], s1 = s0 + s.ptype_mult[pt];
    // clusters of kSiteCluster sites first: one bound rules out all of them
    for (int cb = s0 - s0 % kSiteCluster; cb < s1; cb += kSiteCluster) {
      if (w.cl_d1 &&
          beyond(w.cl_d1[(long long)sp.unit * w.ncl + cb / kSiteCluster], pmf, tf))
        continue;
      const int lo = max(cb, s0), hi = min(cb + kSiteCluster, s1);
      for (int site = lo; site < hi; ++site) {
        double L2[3], v[3], c0;
        if (!site_search(s, w, sp.unit, site, Ps, pmf, t, tf, L2, v, c0)) continue;
        const double *C = s.psite_pos + 3 * site;
        const double maxr = c0 + t + 2.0 * sqrt(c0 * t);
        for (int nc = 0; nc < s.ncell; ++nc) {
          if (s.csize[nc] > maxr) break;
          const double *R = s.cell + 3 * nc;
          const double dx = v[0] - R[0], dy = v[1] - R[1], dz = v[2] - R[2];
          if (dx * dx + dy * dy + dz * dz > t) continue;
          double X[3];
          for (int x = 0; x < 3; ++x) X[x] = Pt[x] - (C[x] + L2[x] + R[x]);
          if (NUC)
            accumulate_nuclear_q_rt(L, X, mu, nu, w0, Q);
          else
            accumulate_overlap_q_rt(L, X, mu, 1.0, Q);
        }
      }
    }
  }
  const double pref = NUC ? exp(-xi * q.r2) : pow(kPi / z3e, 1.5) * exp(-xi * q.r2);
  hermite_to_sh_rt(la, lb, q.A, q.B, q.a1, q.a2, pref, Q,
                   blk + (long long)tl * w.blk_total + sp.boff);
}

template <bool NUC>
__global__ void __launch_bounds__(128)
    k_prim3c_rt(DevSys s, DevWork w, int beg, int n, const Term3c *terms,
                int nterm, int la, int lb, double *blk) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= (long long)n * nterm) return;
  prim3c_item_rt<NUC>(s, w, beg, n, terms, la, lb, blk, g);
}

// ------------------------------------------------------- work queue --
// Every class of a three-centre build in one persistent launch: the items
// of all classes are numbered one after another, the classes ordered by
// their per-item cost (highest angular momentum first) so that the cheap
// classes fill in behind the expensive ones, and each warp takes the next
// 32 items with one atomicAdd on a counter the host zeroes before the
// launch.  A warp's 32 items are consecutive items of one class (or of two
// at a class boundary), the same groups the per-class launches form, and
// every item writes only its own output block, so the results equal the
// per-class launches bit for bit.  No warp waits on another: a warp leaves
// as soon as the counter has passed the last item.
template <int LA, int LB, bool NUC>
__device__ __noinline__ void prim3c_item_q(const DevSys &s, const DevWork &w, int beg, int n,
                                           const Term3c *terms, double *blk, long long g) {
  prim3c_item<LA, LB, NUC>(s, w, beg, n, terms, blk, g);
}

template <bool NUC>
__global__ void __launch_bounds__(128, 3)
    k_prim3c_queue(DevSys s, DevWork w, Prim3cQueue qc, const Term3c *terms, double *blk,
                   unsigned long long *counter) {
  const int lane = threadIdx.x & 31;
  const long long total = qc.off[qc.ncls];
  while (true) {
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(counter, 32ULL);
    base = __shfl_sync(0xffffffffu, base, 0);
    if ((long long)base >= total) return;
    const long long item = (long long)base + lane;
    if (item >= total) continue;
    int c = 0;
    while (item >= qc.off[c + 1]) ++c;
    const long long g = item - qc.off[c];
    const int beg = qc.beg[c], n = qc.n[c];
    switch (qc.cls[c]) {
#define IMAGO_QC(a, b)                                                 \
  case a * 4 + b:                                                      \
    prim3c_item_q<a, b, NUC>(s, w, beg, n, terms, blk, g);             \
    break;
      IMAGO_QC(0, 0) IMAGO_QC(0, 1) IMAGO_QC(0, 2) IMAGO_QC(1, 0) IMAGO_QC(1, 1)
      IMAGO_QC(1, 2) IMAGO_QC(2, 0) IMAGO_QC(2, 1) IMAGO_QC(2, 2)
#undef IMAGO_QC
      default:
        prim3c_item_rt<NUC>(s, w, beg, n, terms, qc.cls[c] / 4, qc.cls[c] % 4, blk, g);
    }
  }
}

template <int LA, int LB>
static int prim2c_one(const DevSys &s, const DevWork &w, int beg, int end,
                      bool kin, double *blk, cudaStream_t st) {
  const int n = end - beg, tb = 128;
  if (n <= 0) return IMAGO_OK;
  if (kin)
    k_prim2c<LA, LB, true><<<(n + tb - 1) / tb, tb, 0, st>>>(s, w, beg, end, blk);
  else
    k_prim2c<LA, LB, false><<<(n + tb - 1) / tb, tb, 0, st>>>(s, w, beg, end, blk);
  IMAGO_CUDA(cudaGetLastError());
  return IMAGO_OK;
}

TermGroups term_pairs(const Term3c *terms_host, int nterm) {
  TermGroups tg{};
  for (int i = 0; i < nterm;) {
    if (tg.n == kMaxTermGroups) {
      tg.n = 0;
      return tg;
    }
    const int c = (i + 1 < nterm && terms_host[i + 1].ptype == terms_host[i].ptype) ? 2 : 1;
    tg.first[tg.n] = (unsigned short)i;
    tg.count[tg.n] = (unsigned char)c;
    ++tg.n;
    i += c;
  }
  return tg;
}

template <int LA, int LB>
static int prim3c_one(const DevSys &s, const DevWork &w, int beg, int end,
                      const Term3c *terms, int nterm, bool nuc, const TermGroups *tg,
                      double *blk, cudaStream_t st) {
  const int n = end - beg, tb = 128;
  if (n <= 0 || nterm <= 0) return IMAGO_OK;
  // EP classes up to d-p: two terms per thread share the walk (d-d keeps
  // one: its two accumulators would not fit the registers)
  if constexpr (LA + LB <= 3) {
    if (!nuc && tg && tg->n > 0 && tg->n < nterm) {
      const unsigned grid = (unsigned)(((long long)n * tg->n + tb - 1) / tb);
      k_prim3c_pair<LA, LB><<<grid, tb, 0, st>>>(s, w, beg, n, terms, *tg, blk);
      IMAGO_CUDA(cudaGetLastError());
      return IMAGO_OK;
    }
  }
  const long long tot = (long long)n * nterm;
  const unsigned grid = (unsigned)((tot + tb - 1) / tb);
  if (nuc)
    k_prim3c<LA, LB, true><<<grid, tb, 0, st>>>(s, w, beg, n, terms, nterm, blk);
  else
    k_prim3c<LA, LB, false><<<grid, tb, 0, st>>>(s, w, beg, n, terms, nterm, blk);
  IMAGO_CUDA(cudaGetLastError());
  return IMAGO_OK;
}

#define IMAGO_FOR_SPD_CLASSES(M) \
  M(0, 0) M(0, 1) M(0, 2) M(1, 0) M(1, 1) M(1, 2) M(2, 0) M(2, 1) M(2, 2)

int launch_prim3c_count(const DevSys &s, const DevWork &w, const int *cls_beg,
                        const Term3c *terms_dev, int nterm, bool nuclear,
                        unsigned long long *count16, cudaStream_t st) {
#define IMAGO_PC(a, b)                                                               \
  {                                                                                 \
    const int beg = cls_beg[a * 4 + b], n = cls_beg[a * 4 + b + 1] - beg;           \
    if (n > 0 && nterm > 0) {                                                       \
      const unsigned grid = (unsigned)(((long long)n * nterm + 127) / 128);         \
      if (nuclear)                                                                  \
        k_prim3c_count<a, b, true><<<grid, 128, 0, st>>>(s, w, beg, n, terms_dev,   \
                                                         nterm, count16 + a * 4 + b); \
      else                                                                          \
        k_prim3c_count<a, b, false><<<grid, 128, 0, st>>>(s, w, beg, n, terms_dev,  \
                                                          nterm, count16 + a * 4 + b); \
      IMAGO_CUDA(cudaGetLastError());                                               \
    }                                                                               \
  }
  IMAGO_FOR_SPD_CLASSES(IMAGO_PC)
#undef IMAGO_PC
  return IMAGO_OK;
}

int launch_prim2c(const DevSys &s, const DevWork &w, const int *cls_beg,
                  int op, double *blk, cudaStream_t st) {
  int rc = IMAGO_OK;
  if (op == kPrim2cMassVel) {
#define IMAGO_MV(a, b)                                                        \
  {                                                                          \
    const int beg = cls_beg[a * 4 + b], n = cls_beg[a * 4 + b + 1] - beg;    \
    if (n > 0) {                                                             \
      k_prim_mv<a, b><<<(n + 127) / 128, 128, 0, st>>>(s, w, beg, beg + n, blk); \
      IMAGO_CUDA(cudaGetLastError());                                        \
    }                                                                        \
  }
    IMAGO_FOR_SPD_CLASSES(IMAGO_MV)
#undef IMAGO_MV
    for (int c = 0; c < 16; ++c) {
      const int la = c / 4, lb = c % 4;
      if (la < 3 && lb < 3) continue;
      const int beg = cls_beg[c], n = cls_beg[c + 1] - beg;
      if (n <= 0) continue;
      k_prim_mv_rt<<<(n + 127) / 128, 128, 0, st>>>(s, w, beg, beg + n, la, lb, blk);
      IMAGO_CUDA(cudaGetLastError());
    }
    return IMAGO_OK;
  }
  const bool kinetic = op == kPrim2cKinetic;
#define IMAGO_P2(a, b)                                                       \
  if (rc == IMAGO_OK)                                                       \
    rc = prim2c_one<a, b>(s, w, cls_beg[a * 4 + b], cls_beg[a * 4 + b + 1], \
                          kinetic, blk, st);
  IMAGO_FOR_SPD_CLASSES(IMAGO_P2)
#undef IMAGO_P2
  for (int c = 0; c < 16 && rc == IMAGO_OK; ++c) {
    const int la = c / 4, lb = c % 4;
    if (la < 3 && lb < 3) continue;
    const int beg = cls_beg[c], end = cls_beg[c + 1], n = end - beg;
    if (n <= 0) continue;
    if (kinetic)
      k_prim2c_rt<true><<<(n + 127) / 128, 128, 0, st>>>(s, w, beg, end, la, lb, blk);
    else
      k_prim2c_rt<false><<<(n + 127) / 128, 128, 0, st>>>(s, w, beg, end, la, lb, blk);
    IMAGO_CUDA(cudaGetLastError());
  }
  return rc;
}

int launch_prim2c_vec(const DevSys &s, const DevWork &w, const int *cls_beg,
                      bool dipole, const double center[3], double *blk,
                      cudaStream_t st) {
  const double3 c3 = make_double3(center ? center[0] : 0.0, center ? center[1] : 0.0,
                                  center ? center[2] : 0.0);
#define IMAGO_PV(a, b)                                                         \
  {                                                                           \
    const int beg = cls_beg[a * 4 + b], n = cls_beg[a * 4 + b + 1] - beg;     \
    if (n > 0) {                                                              \
      const unsigned grid = (n + 127) / 128;                                  \
      if (dipole)                                                             \
        k_prim_vec<a, b, true><<<grid, 128, 0, st>>>(s, w, beg, beg + n, c3, blk);  \
      else                                                                    \
        k_prim_vec<a, b, false><<<grid, 128, 0, st>>>(s, w, beg, beg + n, c3, blk); \
      IMAGO_CUDA(cudaGetLastError());                                         \
    }                                                                         \
  }
  IMAGO_FOR_SPD_CLASSES(IMAGO_PV)
#undef IMAGO_PV
  for (int c = 0; c < 16; ++c) {
    const int la = c / 4, lb = c % 4;
    if (la < 3 && lb < 3) continue;
    const int beg = cls_beg[c], n = cls_beg[c + 1] - beg;
    if (n <= 0) continue;
    const unsigned grid = (n + 127) / 128;
    if (dipole)
      k_prim_vec_rt<true><<<grid, 128, 0, st>>>(s, w, beg, beg + n, la, lb, c3, blk);
    else
      k_prim_vec_rt<false><<<grid, 128, 0, st>>>(s, w, beg, beg + n, la, lb, c3, blk);
    IMAGO_CUDA(cudaGetLastError());
  }
  return IMAGO_OK;
}

int launch_prim3c_ham(const DevSys &s, const DevWork &w, const int *cls_beg,
                      const Term3c *terms_dev, int nterm, const double *coef,
                      int lanes, double *H, cudaStream_t st) {
  if (nterm <= 0) return IMAGO_OK;
  if (lanes != 1 && lanes != 4) return IMAGO_ERR_INVALID;
#define IMAGO_PH(a, b)                                                          \
  {                                                                            \
    const int beg = cls_beg[a * 4 + b], n = cls_beg[a * 4 + b + 1] - beg;      \
    if (n > 0) {                                                               \
      const long long nt = (long long)n * lanes;                               \
      const unsigned grid = (unsigned)((nt + 127) / 128);                      \
      if (lanes == 4)                                                          \
        k_prim3c_ham<a, b, 4><<<grid, 128, 0, st>>>(s, w, beg, n, terms_dev,   \
                                                    nterm, coef, H);           \
      else                                                                     \
        k_prim3c_ham<a, b, 1><<<grid, 128, 0, st>>>(s, w, beg, n, terms_dev,   \
                                                    nterm, coef, H);           \
      IMAGO_CUDA(cudaGetLastError());                                          \
    }                                                                          \
  }
  IMAGO_FOR_SPD_CLASSES(IMAGO_PH)
#undef IMAGO_PH
  for (int c = 0; c < 16; ++c) {
    const int la = c / 4, lb = c % 4;
    if (la < 3 && lb < 3) continue;
    const int beg = cls_beg[c], n = cls_beg[c + 1] - beg;
    if (n <= 0) continue;
    k_prim3c_ham_rt<<<(n + 127) / 128, 128, 0, st>>>(s, w, beg, n, terms_dev, nterm,
                                                     coef, la, lb, H);
    IMAGO_CUDA(cudaGetLastError());
  }
  return IMAGO_OK;
}

// K-overlap: for the three wave vectors, the real and imaginary blocks of
// each shell pair as terms 2 axis and 2 axis + 1.
__global__ void __launch_bounds__(128)
    k_prim_kov(DevSys s, DevWork w, int beg, int end, int la, int lb, KovWaves dk,
               double *blk) {
  const int g = beg + blockIdx.x * blockDim.x + threadIdx.x, ax = blockIdx.y;
  if (g >= end) return;
  const DSp sp = w.sps[w.sp_by_cls[g]];
  const SpGeom q = sp_geom(s, w, sp);
  prim_kov(la, lb, q.a1, q.a2, q.A, q.B, dk.q + 3 * ax,
           blk + (long long)(2 * ax) * w.blk_total + sp.boff,
           blk + (long long)(2 * ax + 1) * w.blk_total + sp.boff);
}

template <int LA, int LB>
__global__ void __launch_bounds__(128)
    k_prim_kov_t(DevSys s, DevWork w, int beg, int end, KovWaves dk, double *blk) {
  const int g = beg + blockIdx.x * blockDim.x + threadIdx.x, ax = blockIdx.y;
  if (g >= end) return;
  const DSp sp = w.sps[w.sp_by_cls[g]];
  const SpGeom q = sp_geom(s, w, sp);
  prim_kov_t<LA, LB>(q.a1, q.a2, q.A, q.B, dk.q + 3 * ax,
                     blk + (long long)(2 * ax) * w.blk_total + sp.boff,
                     blk + (long long)(2 * ax + 1) * w.blk_total + sp.boff);
}

// One thread per (shell pair, wave vector): s, p and d classes unrolled,
// f classes through the runtime routine.
int launch_prim_kov(const DevSys &s, const DevWork &w, const int *cls_beg,
                    const KovWaves &dk, double *blk, cudaStream_t st) {
  for (int c = 0; c < 16; ++c) {
    const int beg = cls_beg[c], n = cls_beg[c + 1] - beg;
    if (n <= 0) continue;
    const dim3 grid((n + 127) / 128, 3);
    switch (c) {
#define IMAGO_KOV(a, b)                                                                 \
  case a * 4 + b:                                                                       \
    k_prim_kov_t<a, b><<<grid, 128, 0, st>>>(s, w, beg, beg + n, dk, blk);              \
    break;
      IMAGO_FOR_SPD_CLASSES(IMAGO_KOV)
#undef IMAGO_KOV
      default:
        k_prim_kov<<<grid, 128, 0, st>>>(s, w, beg, beg + n, c / 4, c % 4, dk, blk);
    }
    IMAGO_CUDA(cudaGetLastError());
  }
  return IMAGO_OK;
}

int launch_prim3c_queue(const DevSys &s, const DevWork &w, const int *cls_beg,
                        const Term3c *terms_dev, int nterm, bool nuclear, double *blk,
                        unsigned long long *counter, int ctas, cudaStream_t st) {
  if (nterm <= 0) return IMAGO_OK;
  Prim3cQueue qc{};
  // highest l_a + l_b first, then the larger l_a
  int order[16], m = 0;
  for (int L = 6; L >= 0; --L)
    for (int la = 3; la >= 0; --la) {
      const int lb = L - la;
      if (lb < 0 || lb > 3) continue;
      order[m++] = la * 4 + lb;
    }
  long long off = 0;
  for (int i = 0; i < m; ++i) {
    const int c = order[i];
    const int n = cls_beg[c + 1] - cls_beg[c];
    if (n <= 0) continue;
    qc.cls[qc.ncls] = c;
    qc.beg[qc.ncls] = cls_beg[c];
    qc.n[qc.ncls] = n;
    qc.off[qc.ncls] = off;
    off += (long long)n * nterm;
    ++qc.ncls;
  }
  qc.off[qc.ncls] = off;
  if (off == 0) return IMAGO_OK;
  IMAGO_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st));
  const long long need = (off + 127) / 128;
  const unsigned grid = (unsigned)std::max<long long>(1, std::min<long long>(ctas, need));
  if (nuclear)
    k_prim3c_queue<true><<<grid, 128, 0, st>>>(s, w, qc, terms_dev, blk, counter);
  else
    k_prim3c_queue<false><<<grid, 128, 0, st>>>(s, w, qc, terms_dev, blk, counter);
  IMAGO_CUDA(cudaGetLastError());
  return IMAGO_OK;
}

int prim3c_queue_ctas_per_sm() {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_prim3c_queue<false>, 128, 0) !=
      cudaSuccess) {
    cudaGetLastError();
    return 1;
  }
  int m = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&m, k_prim3c_queue<true>, 128, 0) !=
      cudaSuccess) {
    cudaGetLastError();
    return std::max(1, n);
  }
  return std::max(1, std::min(n, m));
}

int launch_prim3c(const DevSys &s, const DevWork &w, const int *cls_beg,
                  const Term3c *terms_dev, int nterm, bool nuclear,
                  double *blk, cudaStream_t st, const Term3c *terms_host) {
  int rc = IMAGO_OK;
  TermGroups tg{};
  if (!nuclear && terms_host) tg = term_pairs(terms_host, nterm);
#define IMAGO_P3(a, b)                                                        \
  if (rc == IMAGO_OK)                                                        \
    rc = prim3c_one<a, b>(s, w, cls_beg[a * 4 + b], cls_beg[a * 4 + b + 1],  \
                          terms_dev, nterm, nuclear, &tg, blk, st);
  IMAGO_FOR_SPD_CLASSES(IMAGO_P3)
#undef IMAGO_P3
  for (int c = 0; c < 16 && rc == IMAGO_OK; ++c) {
    const int la = c / 4, lb = c % 4;
    if (la < 3 && lb < 3) continue;
    const int beg = cls_beg[c], end = cls_beg[c + 1], n = end - beg;
    if (n <= 0 || nterm <= 0) continue;
    const long long tot = (long long)n * nterm;
    const unsigned grid = (unsigned)((tot + 127) / 128);
    if (nuclear)
      k_prim3c_rt<true><<<grid, 128, 0, st>>>(s, w, beg, n, terms_dev, nterm, la, lb, blk);
    else
      k_prim3c_rt<false><<<grid, 128, 0, st>>>(s, w, beg, n, terms_dev, nterm, la, lb, blk);
    IMAGO_CUDA(cudaGetLastError());
  }
  return rc;
}

// ------------------------------------------------------- site images --
__global__ void k_site_images(DevSys s, DevWork w, SiteImage *simg) {
  const long long n = (long long)w.nunits * s.nps;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    simg[i] = site_image(s, w, (int)(i / s.nps), (int)(i % s.nps));
}

__global__ void k_cluster_bounds(DevSys s, DevWork w, const SiteImage *simg,
                                 float *cl_d1) {
  const long long n = (long long)w.nunits * w.ncl;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int unit = (int)(i / w.ncl), c = (int)(i % w.ncl);
    const int hi = min((c + 1) * kSiteCluster, s.nps);
    float d = 3.0e38f;
    for (int site = c * kSiteCluster; site < hi; ++site)
      d = fminf(d, simg[(long long)unit * s.nps + site].d1);
    cl_d1[i] = d;
  }
}

// For each unit and potential type, the type's sites in ascending order
// of d1, the lower bound of their distance from the unit's midpoint, as
// offsets within the type (ties by site index).  One warp per (unit, type),
// each lane ranking its sites by counting the smaller ones.
__global__ void k_site_rank(DevSys s, DevWork w, const SiteImage *simg, int *rank) {
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  const int lane = threadIdx.x & 31;
  const long long n = (long long)w.nunits * s.npt;
  for (long long i = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; i < n;
       i += nw) {
    const int unit = (int)(i / s.npt), pt = (int)(i % s.npt);
    const int s0 = s.ptype_first_site[pt], m = s.ptype_mult[pt];
    const SiteImage *si = simg + (long long)unit * s.nps + s0;
    int *out = rank + (long long)unit * s.nps + s0;
    for (int r = lane; r < m; r += 32) {
      const float d = si[r].d1;
      int pos = 0;
      for (int q = 0; q < m; ++q) {
        const float e = si[q].d1;
        pos += (e < d) || (e == d && q < r);
      }
      out[pos] = r;
    }
  }
}

int launch_site_images(const DevSys &s, const DevWork &w, SiteImage *simg,
                       float *cl_d1, cudaStream_t st) {
  const long long n = (long long)w.nunits * s.nps;
  if (n == 0) return IMAGO_OK;
  k_site_images<<<(unsigned)std::min<long long>((n + 255) / 256, 148 * 16), 256,
                  0, st>>>(s, w, simg);
  IMAGO_CUDA(cudaGetLastError());
  const long long nc = (long long)w.nunits * w.ncl;
  if (cl_d1 && nc > 0) {
    k_cluster_bounds<<<(unsigned)std::min<long long>((nc + 255) / 256, 148 * 16),
                       256, 0, st>>>(s, w, simg, cl_d1);
    IMAGO_CUDA(cudaGetLastError());
  }
  const long long nr = (long long)w.nunits * s.npt;
  if (w.site_rank && nr > 0) {
    k_site_rank<<<(unsigned)std::min<long long>((nr + 7) / 8, 148 * 16), 256, 0, st>>>(
        s, w, simg, const_cast<int *>(w.site_rank));
    IMAGO_CUDA(cudaGetLastError());
  }
  return IMAGO_OK;
}

}  // namespace imago
