// scf.cu -- the SCF set-up after the integrals and the potential update of
// every SCF iteration (makeSCFPot), on the device where the work scales
// with the system.
//
// Set-up (imago_scf_create), once per structure:
//   * lattice lists: the real list of the integrals and the reciprocal list
//     (initializeLattice, lattice.f90:310-444, negligLimitRecip =
//     4 logElecThresh minPotAlpha);
//   * electrostatic operators (neutralAndNuclearQPot, elecStat.f90:59-664;
//     residualQ, elecStat.f90:666-1042): k_es_pairs evaluates every
//     (site i, site j) pair over the real lattice (one CTA per pair, one
//     thread per alpha pair, the cells in the reference's order) and
//     k_res_pairs the reciprocal sum; k_es_reduce adds the pairs into the
//     per-type blocks in the reference's site order;
//   * exchange-correlation mesh (getECMeshParameters /
//     makeECMeshAndOverlap, exchCorr.f90:63-873): the rays and their
//     weights on the host, the operator exchRhoOp(term, point) = sum over
//     sites and cells of exp(-alpha r^2) by k_xc_operator (one thread per
//     (point, potential type)), and its overlap by k_xc_overlap;
//   * core charge fit (makeCoreRho, coreCharge.f90:27-578) and the
//     integration constants (potential.f90:149-160) on the host.
//
// Update (imago_scf_pot_update), per iteration: the potDim x potDim fits
// and the mixing of makeSCFPot (potentialUpdate.F90:53-1866) on the host
// (potDim <= 64: tens of microseconds), the charge on the mesh, the local
// density functional and the fitted exchange-correlation potential on the
// device (k_xc_points, k_xc_accum, k_reduce_chunks), and the real-space
// convergence measure per site (k_xc_delta).
//
// Scope: spin 1, rel 0, LDA (XC_CODE 100, 101, 102), no +UJ.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

#include "intg.cuh"
#include "lattice.cuh"
#include "../../include/imago_scf.h"

namespace {

using namespace imago;

constexpr int kMaxPotAlphas = 32;
constexpr int kEsThreads = 256;
constexpr int kEsChunk = 256;
constexpr int kResThreads = 64;
constexpr int kResPhaseChunk = 1024;
constexpr int kChunkPoints = 512;

// error_fn (mathSubs.f90:22-140): the reference's rational approximation of
// erf (W. J. Cody's, as in the Sandia library it cites), kept so that the
// electrostatic operators round as the reference's do.
__host__ __device__ inline double ref_erf(double x) {
  const double ax = fabs(x);
  if (ax > 6.0) return x / ax;
  const double x2 = ax * ax;
  if (ax <= 0.46875) {
    double a = ax * (242.6679552305318 +
                     x2 * (21.97926161829415 + x2 * (6.996383488619136 +
                                                      x2 * -0.03560984370181539)));
    a = a / (215.0588758698612 +
             x2 * (91.16490540451490 + x2 * (15.08279763040779 + x2 * 1.0)));
    return x < 0.0 ? -a : a;
  }
  double a;
  if (ax <= 4.0) {
    a = exp(-x2) *
        (22.898992851659 +
         ax * (26.094746956075 +
               ax * (14.571898596926 +
                     ax * (4.2677201070898 + ax * (0.56437160686381 +
                                                   ax * -0.0000060858151959688)))));
    a = a / (22.898985749891 +
             ax * (51.933570687552 +
                   ax * (50.273202863803 +
                         ax * (26.288795758761 + ax * (7.5688482293618 + ax * 1.0)))));
  } else {
    const double inv = 1.0 / x2;
    a = inv * (-0.0121308276389978 +
               inv * (-0.119903955268146 +
                      inv * (-0.243911029488626 + inv * -0.0324319519277746)));
    a = a / (0.043002664345277 +
             inv * (0.489552441961437 + inv * (1.43771227937118 + inv * 1.0)));
    a = exp(-x2) * (0.564189583547756 + a) / ax;
  }
  return copysign(1.0 - a, x);
}

// Single-precision (default REAL) literals of the functionals, as gfortran
// stores them.
__host__ __device__ constexpr double f32(float v) { return (double)v; }

// wignerXC / wignerXCEnergy (potentialUpdate.F90:2835-2894).
__device__ inline void wigner_xc(double rho, double &pot, double &en) {
  const double r13 = pow(rho, 0.3333333333333333333);
  const double f = 1.0 + 12.57 * r13;
  pot = -r13 * (0.984 + (0.943656 + 8.8963 * r13) / (f * f));
  en = -0.738 * r13 * (1.0 + 0.959 / f);
}
__device__ inline double wigner_xc_energy(double rho) {
  const double r13 = pow(rho, 0.3333333333333333333);
  return -0.738 * r13 * (1.0 + 0.959 / (1.0 + 12.57 * r13));
}

// ceperleyAlderXC / ceperleyAlderXCEnergy (potentialUpdate.F90:2898-3031),
// the Perdew-Zunger form; the parameters are single-precision literals.
__device__ inline void ceperley_alder(double rho, double &pot, double &en) {
  if (rho < kSmallThresh) {
    pot = en = 0.0;
    return;
  }
  const double third = f32(0.33333333f);
  const double alpha = pow(4.0 / (9.0 * kPi), third);
  const double rs = pow(3.0 / (4.0 * kPi * rho), third);
  const double ex0 = 3.0 / (2.0 * kPi * alpha);
  const double ex = -ex0 / rs;
  if (rs >= 1.0) {
    const double g = f32(-0.1423f), b1 = f32(1.0529f), b2 = f32(0.3334f);
    const double sq = sqrt(rs);
    const double ec = g / (1 + b1 * sq + b2 * rs);
    en = ex + ec;
    pot = f32(4.0f / 3.0f) * ex +
          ec * ec / g * (1 + f32(7.0f / 6.0f) * b1 * sq + f32(4.0f / 3.0f) * b2 * rs);
  } else {
    const double af = f32(0.0311f), bf = f32(-0.0480f), cf = f32(0.0020f),
                 df = f32(-0.0116f);
    const double ln = log(rs);
    en = ex + af * ln + bf + cf * rs * ln + df * rs;
    pot = f32(4.0f / 3.0f) * ex + af * ln + (bf - f32(1.0f / 3.0f) * af) +
          f32(2.0f / 3.0f) * cf * rs * ln + f32(1.0f / 3.0f) * (2 * df - cf) * rs;
  }
  pot = pot * f32(0.5f);
  en = en * f32(0.5f);
}

// hedinLundqvistXC / hedinLundqvistXCEnergy (potentialUpdate.F90:3033-3123).
__device__ inline void hedin_lundqvist(double rho, double &pot, double &en) {
  if (rho < kSmallThresh) {
    pot = en = 0.0;
    return;
  }
  const double third = f32(0.33333333f);
  const double alpha = pow(4.0 / (9.0 * kPi), third);
  const double rs = pow(3.0 / (4.0 * kPi * rho), third);
  const double x = rs / 21.0;
  const double lg = log(1.0 + 1.0 / x);
  pot = (-2.0 / (kPi * alpha * rs) - 0.045 * lg) * f32(0.5f);
  en = (-0.75 * 2.0 / (kPi * alpha * rs) -
        0.045 * ((1 + pow(x, 3.0)) * lg + x / 2.0 - pow(x, 2.0) - third)) *
       f32(0.5f);
}

// ------------------------------------------------------------ device data

struct ScfDev {
  int nps, npt, pot_dim;
  double Te;                      // logElecThresh
  double rv[9], inv[9];
  const int *ps_type;             // 0-based
  const double *ps_pos;           // [site][3]
  const int *pt_off, *pt_n;       // per type: first term, number of alphas
  const double *pt_z, *pt_nuc;    // nucCharge, nucAlpha
  const double *alpha;            // [potDim]
  int ncell;
  const double *cell, *csize;
  int nrecip;
  const double *rcell;            // [G][3]
};

// Nearest lattice vector (the role of findLatticeVector, lattice.f90:784-888):
// rounded fractional coordinates and their 26 neighbours.
__host__ __device__ inline void nearest_vec(const double *rv, const double *inv,
                                            const double v[3], double out[3]) {
  double base[3] = {0.0, 0.0, 0.0};
  for (int i = 0; i < 3; ++i) {
    const double f = v[0] * inv[3 * i] + v[1] * inv[3 * i + 1] + v[2] * inv[3 * i + 2];
    double r = (double)(long long)(fabs(f) + 0.5);
    if (f < 0.0) r = -r;
    for (int x = 0; x < 3; ++x) base[x] += rv[3 * i + x] * r;
  }
  double best[3] = {base[0], base[1], base[2]};
  double bd = 0.0;
  for (int x = 0; x < 3; ++x) bd += (v[x] - base[x]) * (v[x] - base[x]);
  for (int i = -1; i <= 1; ++i)
    for (int j = -1; j <= 1; ++j)
      for (int k = -1; k <= 1; ++k) {
        if (!i && !j && !k) continue;
        double c[3], d = 0.0;
        for (int x = 0; x < 3; ++x) {
          c[x] = base[x] + i * rv[x] + j * rv[3 + x] + k * rv[6 + x];
          d += (v[x] - c[x]) * (v[x] - c[x]);
        }
        if (d < bd * (1.0 - 1e-12)) {
          bd = d;
          best[0] = c[0];
          best[1] = c[1];
          best[2] = c[2];
        }
      }
  out[0] = best[0];
  out[1] = best[1];
  out[2] = best[2];
}

// --------------------------------------------------- electrostatic pairs

// One CTA per (site i, site j): the neutral-charge operators, the overlap
// of the potential Gaussians and the screened nuclear potential
// (neutralAndNuclearQPot, elecStat.f90:249-520).  A thread owns up to
// kMaxPotAlphas^2 / kEsThreads entries (a, b), a over the alphas of i's type
// and b over j's, and walks the cells in order; per cell, the alpha pairs
// whose smaller index reaches the reference's first diagonal that fails the
// range test are skipped (the reference leaves its alpha loop there).  The
// cells are screened in chunks first: a cell that fails the test of the two
// most diffuse alphas and of the most diffuse nuclear term contributes
// nothing.  Output per pair: [3][n1][n2] (non-local neutral, local
// neutral, overlap), then [n1] of the nuclear term.
__global__ void __launch_bounds__(kEsThreads)
k_es_pairs(ScfDev s, const double *minsep, long long pair_stride, double *out) {
  const int pair = blockIdx.x;
  const int i = pair / s.nps, j = pair % s.nps;
  const int t1 = s.ps_type[i], t2 = s.ps_type[j];
  const int n1 = s.pt_n[t1], n2 = s.pt_n[t2];
  const double *a1 = s.alpha + s.pt_off[t1], *a2 = s.alpha + s.pt_off[t2];
  const int nmin = min(n1, n2);
  const double T = s.Te;
  const double sep[3] = {minsep[3 * pair], minsep[3 * pair + 1], minsep[3 * pair + 2]};
  const double nuc = s.pt_nuc[t2], z2 = s.pt_z[t2];
  constexpr int kPer = kMaxPotAlphas * kMaxPotAlphas / kEsThreads;
  double nl[kPer], loc[kPer], ol[kPer];
  int ea[kPer], eb[kPer], el[kPer];
  double rpa[kPer], rpas[kPer], s1[kPer], nq[kPer], oc[kPer];
  const int ne = n1 * n2;
#pragma unroll
  for (int q = 0; q < kPer; ++q) {
    nl[q] = loc[q] = ol[q] = 0.0;
    const int e = threadIdx.x + q * kEsThreads;
    ea[q] = e < ne ? e / n2 : -1;
    eb[q] = e < ne ? e % n2 : 0;
    if (ea[q] >= 0) {
      const double x1 = a1[ea[q]], x2 = a2[eb[q]];
      rpa[q] = x1 * x2 / (x1 + x2);
      rpas[q] = sqrt(rpa[q]);
      s1[q] = sqrt(x1);
      nq[q] = kPi * kPi * kPi / (x1 * s1[q] * x2 * sqrt(x2));
      oc[q] = pow(kPi / (x1 + x2), 1.5);
      // the diagonals l = 0 .. el that must pass for this entry to count
      el[q] = min(min(ea[q], eb[q]), nmin - 2);
    }
  }
  // the nuclear term of alpha a = threadIdx.x
  double nucsum = 0.0;
  const bool nuc_thread = threadIdx.x < n1;
  const double na = nuc_thread ? a1[threadIdx.x] : 1.0;
  const double nf = na + nuc;
  __shared__ int act[kEsChunk];
  __shared__ int nact;
  const double rpa00 = a1[0] * a2[0] / (a1[0] + a2[0]);
  for (int c0 = 0; c0 < s.ncell; c0 += kEsChunk) {
    if (threadIdx.x == 0) nact = 0;
    __syncthreads();
    // ordered compaction of the chunk's cells that can contribute
    const int c = c0 + threadIdx.x;
    bool live = false;
    if (c < s.ncell) {
      double r2 = 0.0;
      for (int x = 0; x < 3; ++x) {
        const double d = sep[x] - s.cell[3 * c + x];
        r2 += d * d;
      }
      live = nmin < 2 || !(rpa00 * r2 > T) ||
             (r2 * a1[0] * nuc / (a1[0] + nuc) < T);
    }
    const unsigned ball = __ballot_sync(0xffffffffu, live);
    __shared__ int wcount[kEsThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) wcount[warp] = __popc(ball);
    __syncthreads();
    if (live) {
      int base = 0;
      for (int w = 0; w < warp; ++w) base += wcount[w];
      act[base + __popc(ball & ((1u << lane) - 1u))] = c;
    }
    if (threadIdx.x == 0) {
      int tot = 0;
      for (int w = 0; w < kEsThreads / 32; ++w) tot += wcount[w];
      nact = tot;
    }
    __syncthreads();
    for (int q0 = 0; q0 < nact; ++q0) {
      const int cc = act[q0];
      double r2 = 0.0;
      for (int x = 0; x < 3; ++x) {
        const double d = sep[x] - s.cell[3 * cc + x];
        r2 += d * d;
      }
      const double r = sqrt(r2);
#pragma unroll
      for (int q = 0; q < kPer; ++q) {
        if (ea[q] < 0) continue;
        bool in = true;
        for (int l = 0; l <= el[q]; ++l) {
          const double rl = a1[l] * a2[l] / (a1[l] + a2[l]);
          if (rl * r2 > T) {
            in = false;
            break;
          }
        }
        if (!in) continue;
        if (fabs(r2) >= kSmallThresh) {
          nl[q] = nl[q] + nq[q] / r * (-ref_erf(s1[q] * r) + ref_erf(rpas[q] * r));
        } else {
          loc[q] = loc[q] + nq[q] * (2.0 / sqrt(kPi)) * rpas[q];
        }
        ol[q] = ol[q] + oc[q] * exp(-rpa[q] * r2);
      }
      if (nuc_thread) {
        // alphas 0 .. threadIdx.x all inside the nuclear screen
        bool in = true;
        double scr = 0.0;
        for (int m = 0; m <= (int)threadIdx.x; ++m) {
          const double am = a1[m];
          scr = r2 * am * nuc / (am + nuc);
          if (!(scr < T)) {
            in = false;
            break;
          }
        }
        if (in) {
          if (fabs(scr) >= kSmallThresh) {
            const double co = na * r / sqrt(nf);
            nucsum = nucsum - z2 * pow(kPi, 1.5) * exp(-scr) * ref_erf(co) / co / nf;
          } else {
            nucsum = nucsum - z2 * exp(-scr) * (2.0 * kPi) / nf;
          }
        }
      }
    }
    __syncthreads();
  }
  double *o = out + pair * pair_stride;
  const int blk = kMaxPotAlphas * kMaxPotAlphas;
#pragma unroll
  for (int q = 0; q < kPer; ++q) {
    if (ea[q] < 0) continue;
    const int e = ea[q] * n2 + eb[q];
    o[e] = nl[q];
    o[blk + e] = loc[q];
    o[2 * blk + e] = ol[q];
  }
  if (nuc_thread) o[3 * blk + threadIdx.x] = nucsum;
}

// residualQ (elecStat.f90:794-1005), one CTA per (site i, site j), one thread
// per alpha k of i's type: the real-space part over the cells in order
// until the first cell beyond both ranges, then the reciprocal sum
// sum_{G != 0} exp(-G^2 / (4 mu_k)) / G^2 cos(G . (pos_i - pos_j)), the
// cosines staged in shared memory.  rce [table][G][kMaxPotAlphas] holds
// exp(-G^2/(4 mu_k))/G^2; mra_sqrt [table][kMaxPotAlphas] sqrt(mu_k).
__global__ void __launch_bounds__(kResThreads)
k_res_pairs(ScfDev s, const double *minsep, const int *table_of_type, const double *rce,
            const double *mra_sqrt, double min_pot_alpha, double volume, double *out) {
  const int pair = blockIdx.x;
  const int i = pair / s.nps, j = pair % s.nps;
  const int t1 = s.ps_type[i], t2 = s.ps_type[j];
  const int n1 = s.pt_n[t1];
  const double *a1 = s.alpha + s.pt_off[t1];
  const double a21 = s.alpha[s.pt_off[t2]];
  const int tab = table_of_type[t1];
  const int k = threadIdx.x;
  const bool on = k < n1;
  const double sqT = sqrt(s.Te);
  const double sep[3] = {minsep[3 * pair], minsep[3 * pair + 1], minsep[3 * pair + 2]};
  double acc = 0.0;
  double mra = 0.0;
  double af = 0.0, rps = 0.0;
  if (on) {
    const double x1 = a1[k];
    const double f1 = pow(kPi, 1.5) / (x1 * sqrt(x1));
    const double f2 = pow(kPi, 1.5) / (a21 * sqrt(a21));
    af = f1 * f2;
    rps = sqrt(x1 * a21 / (x1 + a21));
    mra = mra_sqrt[tab * kMaxPotAlphas + k];
    const double self = 2.0 / sqrt(kPi) * af * (rps - mra);
    for (int c = 0; c < s.ncell; ++c) {
      double r2 = 0.0;
      for (int x = 0; x < 3; ++x) {
        const double d = sep[x] - s.cell[3 * c + x];
        r2 += d * d;
      }
      if (r2 < kSmallThresh) {
        acc = acc + self;
      } else {
        const double r = sqrt(r2);
        if (mra * r > sqT && rps * r > sqT) break;
        acc = acc + af * (-ref_erf(mra * r) + ref_erf(rps * r)) / r;
      }
    }
  }
  // raw separation for the reciprocal phases
  double raw[3];
  for (int x = 0; x < 3; ++x) raw[x] = s.ps_pos[3 * i + x] - s.ps_pos[3 * j + x];
  __shared__ double ph[kResPhaseChunk];
  double rs = 0.0;
  for (int g0 = 1; g0 < s.nrecip; g0 += kResPhaseChunk) {
    const int gn = min(kResPhaseChunk, s.nrecip - g0);
    for (int q = threadIdx.x; q < gn; q += blockDim.x) {
      const double *G = s.rcell + 3 * (g0 + q);
      ph[q] = cos(G[0] * raw[0] + G[1] * raw[1] + G[2] * raw[2]);
    }
    __syncthreads();
    if (on) {
      const double *tb = rce + ((long long)tab * s.nrecip + g0) * kMaxPotAlphas + k;
      for (int q = 0; q < gn; ++q) rs = rs + tb[(long long)q * kMaxPotAlphas] * ph[q];
    }
    __syncthreads();
  }
  if (on) {
    const double vf = 4.0 * kPi * af / volume;
    acc = acc + vf * (rs - 0.25 / min_pot_alpha);
    out[(long long)pair * kMaxPotAlphas + k] = acc;
  }
}

// Per-type blocks from the pair partials, added over the site pairs in the
// reference's order (i over the sites of the column's type, then j over the
// sites of the row's type).  One thread per output element.
__global__ void k_es_reduce(ScfDev s, const double *part, long long pair_stride,
                            const double *res_part, double *nl, double *loc, double *ol,
                            double *nlnuc, double *nlres, int ntypes) {
  const int P = s.pot_dim;
  const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int blk = kMaxPotAlphas * kMaxPotAlphas;
  // the term's type and alpha index
  auto type_of = [&](int term, int &t, int &a) {
    for (t = 0; t < ntypes; ++t)
      if (term < s.pt_off[t] + s.pt_n[t]) break;
    a = term - s.pt_off[t];
  };
  if (idx < (long long)P * P) {
    const int row = (int)(idx % P), col = (int)(idx / P);
    int t1, a, t2, b;
    type_of(col, t1, a);
    type_of(row, t2, b);
    const int n2 = s.pt_n[t2];
    double x = 0.0, y = 0.0, z = 0.0;
    for (int i = 0; i < s.nps; ++i) {
      if (s.ps_type[i] != t1) continue;
      for (int j = 0; j < s.nps; ++j) {
        if (s.ps_type[j] != t2) continue;
        const double *o = part + (long long)(i * s.nps + j) * pair_stride;
        const int e = a * n2 + b;
        x = x + o[e];
        y = y + o[blk + e];
        z = z + o[2 * blk + e];
      }
    }
    nl[idx] = x;
    loc[idx] = y;
    ol[idx] = z;
    return;
  }
  long long r = idx - (long long)P * P;
  if (r < P) {
    int t1, a;
    type_of((int)r, t1, a);
    double x = 0.0;
    for (int i = 0; i < s.nps; ++i) {
      if (s.ps_type[i] != t1) continue;
      for (int j = 0; j < s.nps; ++j)
        x = x + part[(long long)(i * s.nps + j) * pair_stride + 3 * blk + a];
    }
    nlnuc[r] = x;
    return;
  }
  r -= P;
  if (r < (long long)ntypes * P) {
    const int t2 = (int)(r % ntypes), col = (int)(r / ntypes);
    int t1, a;
    type_of(col, t1, a);
    double x = 0.0;
    for (int i = 0; i < s.nps; ++i) {
      if (s.ps_type[i] != t1) continue;
      for (int j = 0; j < s.nps; ++j) {
        if (s.ps_type[j] != t2) continue;
        x = x + res_part[(long long)(i * s.nps + j) * kMaxPotAlphas + a];
      }
    }
    nlres[r] = x;
  }
}

// ------------------------------------------------- exchange-correlation mesh

// exchRhoOp(term, point) (exchCorr.f90:613-790): one thread per (point,
// potential type): over the sites of the type in order, the nearest-image
// offset of the point, the cells up to the reference's radius in order,
// and the type's alphas until alpha r^2 exceeds logElecThresh.
__global__ void k_xc_operator(ScfDev s, const double *pts, int npts, int ntypes,
                              double *op) {
  const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (id >= (long long)npts * ntypes) return;
  const int p = (int)(id / ntypes), t = (int)(id % ntypes);
  const int n = s.pt_n[t];
  const double *al = s.alpha + s.pt_off[t];
  const double T = s.Te;
  const double neg = T / al[0];
  double acc[kMaxPotAlphas];
  for (int q = 0; q < kMaxPotAlphas; ++q) acc[q] = 0.0;
  const double *x = pts + 3 * (long long)p;
  for (int l = 0; l < s.nps; ++l) {
    if (s.ps_type[l] != t) continue;
    double v[3], L[3], off[3];
    for (int c = 0; c < 3; ++c) v[c] = x[c] - s.ps_pos[3 * l + c];
    nearest_vec(s.rv, s.inv, v, L);
    double m2 = 0.0;
    for (int c = 0; c < 3; ++c) {
      off[c] = v[c] - L[c];
      m2 += off[c] * off[c];
    }
    const double plus = neg + m2 + 2.0 * sqrt(neg * m2);
    for (int m = 0; m < s.ncell; ++m) {
      if (s.csize[m] > plus) break;
      double r2 = 0.0;
      for (int c = 0; c < 3; ++c) {
        const double d = off[c] - s.cell[3 * m + c];
        r2 += d * d;
      }
      if (r2 > neg) continue;
      for (int q = 0; q < n; ++q) {
        const double e = al[q] * r2;
        if (e > T) break;
        acc[q] += exp(-e);
      }
    }
  }
  double *o = op + (long long)p * s.pot_dim + s.pt_off[t];
  for (int q = 0; q < n; ++q) o[q] = acc[q];
}

// Partial sums over chunks of kChunkPoints points of
//   overlap:  op(k, p) op(a, p) w(p) for a <= k   (mode 0, P(P+1)/2 values)
//   update:   g(c, p) op(a, p) for c = 0..2        (mode 1, 3P values)
// one thread per value, the chunk's points in order.
__global__ void k_xc_chunks(const double *op, const double *w, const double *g, int npts,
                            int P, int mode, double *part) {
  const int nval = mode == 0 ? P * (P + 1) / 2 : 3 * P;
  const int chunk = blockIdx.x;
  const int p0 = chunk * kChunkPoints, p1 = min(npts, p0 + kChunkPoints);
  for (int v = threadIdx.x; v < nval; v += blockDim.x) {
    double acc = 0.0;
    if (mode == 0) {
      int k = 0;
      while ((k + 1) * (k + 2) / 2 <= v) ++k;
      const int a = v - k * (k + 1) / 2;
      for (int p = p0; p < p1; ++p) {
        const double *o = op + (long long)p * P;
        acc = acc + o[k] * o[a] * w[p];
      }
    } else {
      const int c = v / P, a = v % P;
      for (int p = p0; p < p1; ++p) acc = acc + g[3 * (long long)p + c] * op[(long long)p * P + a];
    }
    part[(long long)chunk * nval + v] = acc;
  }
}

__global__ void k_reduce_chunks(const double *part, int nchunk, int nval, double *out) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nval) return;
  double acc = 0.0;
  for (int c = 0; c < nchunk; ++c) acc = acc + part[(long long)c * nval + v];
  out[v] = acc;
}

// Charge and functional at every mesh point (potentialUpdate.F90:855-1045):
// one warp per point, the two fitted densities as dot products over the
// terms, clipped at zero, then g(0..2, p) = w_p (v_xc(total), e_xc(total),
// e_xc(core)).
__global__ void k_xc_points(const double *op, const double *w, const double *rho_tot,
                            const double *rho_core, int npts, int P, int xc, double *g) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= npts) return;
  const double *o = op + (long long)warp * P;
  double tot = 0.0, core = 0.0;
  for (int a = lane; a < P; a += 32) {
    tot += o[a] * rho_tot[a];
    core += o[a] * rho_core[a];
  }
  for (int d = 16; d; d >>= 1) {
    tot += __shfl_xor_sync(0xffffffffu, tot, d);
    core += __shfl_xor_sync(0xffffffffu, core, d);
  }
  if (lane) return;
  if (core < 0.0) core = 0.0;
  if (tot < 0.0) tot = 0.0;
  double v1, v2, v3, dummy;
  if (xc == 100) {
    wigner_xc(tot, v1, v2);
    v3 = wigner_xc_energy(core);
  } else if (xc == 101) {
    ceperley_alder(tot, v1, v2);
    ceperley_alder(core, dummy, v3);
  } else {
    hedin_lundqvist(tot, v1, v2);
    hedin_lundqvist(core, dummy, v3);
  }
  const double wp = w[warp];
  g[3 * (long long)warp] = wp * v1;
  g[3 * (long long)warp + 1] = wp * v2;
  g[3 * (long long)warp + 2] = wp * v3;
}

// The real-space measure of the change of the potential per site
// (potentialUpdate.F90:1419-1458): sum_p w_p (sum_a op(a,p) dV_a)^2 and
// sum_p w_p over the site's points, one CTA per site, partial sums added
// in a fixed tree.
__global__ void k_xc_delta(const double *op, const double *w, const int *site_off,
                           const int *site_n, const double *dv, int P, double *out) {
  const int site = blockIdx.x;
  const int n = site_n[site], off = site_off[site];
  double wd = 0.0, ws = 0.0;
  for (int q = threadIdx.x; q < n; q += blockDim.x) {
    const double *o = op + (long long)(off + q) * P;
    double d = 0.0;
    for (int a = 0; a < P; ++a) d += o[a] * dv[a];
    wd += w[off + q] * d * d;
    ws += w[off + q];
  }
  __shared__ double s1[256], s2[256];
  s1[threadIdx.x] = wd;
  s2[threadIdx.x] = ws;
  __syncthreads();
  for (int h = blockDim.x / 2; h; h >>= 1) {
    if (threadIdx.x < h) {
      s1[threadIdx.x] += s1[threadIdx.x + h];
      s2[threadIdx.x] += s2[threadIdx.x + h];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[2 * site] = s1[0];
    out[2 * site + 1] = s2[0];
  }
}

// ------------------------------------------------------------ host math

// dposvx('E', 'U') as solveDPOSVX calls it (interfaces.F90:236-293):
// equilibration by the inverse square roots of the diagonal when the ratio
// of the smallest to the largest is below 0.1, Cholesky of the upper
// triangle, solution, and iterative refinement on the equilibrated system
// while the componentwise backward error halves (at most five steps).  A is
// column-major with leading dimension n; only its upper triangle is read.
int solve_spd(int n, int nrhs, const double *A, double *B) {
  std::vector<double> s(n), a(n * (size_t)n), u(n * (size_t)n, 0.0);
  double smin = 1e308, smax = 0.0;
  for (int i = 0; i < n; ++i) {
    const double d = A[(size_t)i * n + i];
    if (!(d > 0.0)) return IMAGO_ERR_RANGE;
    smin = std::min(smin, d);
    smax = std::max(smax, d);
  }
  const bool equil = std::sqrt(smin) / std::sqrt(smax) < 0.1;
  for (int i = 0; i < n; ++i) s[i] = equil ? 1.0 / std::sqrt(A[(size_t)i * n + i]) : 1.0;
  for (int c = 0; c < n; ++c)
    for (int r = 0; r <= c; ++r) {
      const double v = s[r] * A[(size_t)c * n + r] * s[c];
      a[(size_t)c * n + r] = v;
      a[(size_t)r * n + c] = v;
    }
  // upper Cholesky: a = U^T U
  for (int j = 0; j < n; ++j) {
    double d = a[(size_t)j * n + j];
    for (int k = 0; k < j; ++k) d -= u[(size_t)j * n + k] * u[(size_t)j * n + k];
    if (!(d > 0.0)) return IMAGO_ERR_RANGE;
    const double ujj = std::sqrt(d);
    u[(size_t)j * n + j] = ujj;
    for (int c = j + 1; c < n; ++c) {
      double v = a[(size_t)c * n + j];
      for (int k = 0; k < j; ++k) v -= u[(size_t)j * n + k] * u[(size_t)c * n + k];
      u[(size_t)c * n + j] = v / ujj;
    }
  }
  auto chol_solve = [&](std::vector<double> &x) {
    for (int i = 0; i < n; ++i) {  // U^T y = x
      double v = x[i];
      for (int k = 0; k < i; ++k) v -= u[(size_t)i * n + k] * x[k];
      x[i] = v / u[(size_t)i * n + i];
    }
    for (int i = n - 1; i >= 0; --i) {  // U x = y
      double v = x[i];
      for (int k = i + 1; k < n; ++k) v -= u[(size_t)k * n + i] * x[k];
      x[i] = v / u[(size_t)i * n + i];
    }
  };
  const double eps = 1.1102230246251565e-16;
  for (int r = 0; r < nrhs; ++r) {
    std::vector<double> b(n), x(n), res(n);
    for (int i = 0; i < n; ++i) b[i] = s[i] * B[(size_t)r * n + i];
    x = b;
    chol_solve(x);
    double last = 3.0;
    for (int it = 0; it < 5; ++it) {
      double berr = 0.0;
      for (int i = 0; i < n; ++i) {
        double v = b[i], den = std::fabs(b[i]);
        for (int k = 0; k < n; ++k) {
          v -= a[(size_t)k * n + i] * x[k];
          den += std::fabs(a[(size_t)k * n + i]) * std::fabs(x[k]);
        }
        res[i] = v;
        if (den > 0.0) berr = std::max(berr, std::fabs(v) / den);
      }
      if (!(berr > eps && 2.0 * berr <= last)) break;
      last = berr;
      chol_solve(res);
      for (int i = 0; i < n; ++i) x[i] += res[i];
    }
    for (int i = 0; i < n; ++i) B[(size_t)r * n + i] = s[i] * x[i];
  }
  return IMAGO_OK;
}

double seq_dot(const double *a, const double *b, int n) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) s = s + a[i] * b[i];
  return s;
}

struct PType {
  int n, off, mult, element;
  double z, nucalpha, covrad;
};

}  // namespace

struct imago_scf {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  double rv[9], inv[9], recip[9], volume = 0.0;
  double Tb = 0.0, Te = 0.0, min_pot_alpha = 0.0, min_atom_alpha = 0.0;
  int P = 0, npt = 0, nps = 0;
  std::vector<PType> pt;
  std::vector<double> alpha;   // [P]
  std::vector<int> ps_type;    // 0-based
  std::vector<double> ps_pos;
  std::vector<double> cells, csize, rcells, rcsize;
  // set-up results (column-major potDim x potDim)
  std::vector<double> pot_ol, nl_neut, l_neut, nl_nuc, l_nuc, nl_res, core_rho, xc_ol, intg;
  // mesh
  std::vector<int> site_n, site_off;
  std::vector<double> pts, w;
  int npoints = 0;
  double *d_op = nullptr, *d_w = nullptr, *d_buf = nullptr;
  int *d_site = nullptr;
  size_t buf_doubles = 0;
  // SCF control
  int xc = 100, feedback = 2;
  double relax = 0.2, convg = 1e-4, nelec = 0.0;
  // Anderson history (module arrays xl1, xl2, yl1, yl2 of the reference)
  bool hist = false;
  int iter = 1;
  std::vector<double> xl1, xl2, yl1, yl2;
  float ms[3] = {0, 0, 0};
  ScfDev dev{};
  std::vector<void *> allocs;
};

namespace {

template <class T>
int dalloc(imago_scf *c, T **p, size_t n) {
  void *q = nullptr;
  if (cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    return IMAGO_ERR_NOMEM;
  }
  c->allocs.push_back(q);
  *p = static_cast<T *>(q);
  return IMAGO_OK;
}

template <class T>
int upload(imago_scf *c, const std::vector<T> &v, const T **out) {
  T *p = nullptr;
  int rc = dalloc(c, &p, v.size());
  if (rc) return rc;
  if (!v.empty())
    IMAGO_CUDA(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice,
                               c->stream));
  *out = p;
  return IMAGO_OK;
}

// getRecipCellVectors (lattice.f90:174-236).
void recip_vectors(imago_scf *c) {
  double vol = 0.0;
  for (int i = 0; i < 3; ++i) {
    vol = 0.0;
    const int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
    for (int j = 0; j < 3; ++j) {
      const int j1 = (j + 1) % 3, j2 = (j + 2) % 3;
      c->recip[3 * i + j] = c->rv[3 * i1 + j1] * c->rv[3 * i2 + j2] -
                            c->rv[3 * i1 + j2] * c->rv[3 * i2 + j1];
      vol = vol + c->recip[3 * i + j] * c->rv[3 * i + j];
    }
    for (int j = 0; j < 3; ++j) c->recip[3 * i + j] = 2.0 * kPi * c->recip[3 * i + j] / vol;
  }
  c->volume = std::fabs(vol);
  for (int i = 0; i < 9; ++i) c->inv[i] = c->recip[i] / (2.0 * kPi);
}

int read_system(imago_scf *c, const imago_system *s, const imago_scf_params *p) {
  if (!s || !p || s->num_pot_types <= 0 || s->num_pot_sites <= 0 || !s->pot_type_alphas ||
      !s->pot_type_num_alphas || !s->pot_site_type || !s->pot_site_pos ||
      !p->covalent_radius || !(s->electro_convg > 0.0) || !(s->basis_fn_convg > 0.0))
    return IMAGO_ERR_INVALID;
  if (p->xc_code != 100 && p->xc_code != 101 && p->xc_code != 102) return IMAGO_ERR_RANGE;
  if (p->num_sample_vectors < 2 || p->feedback_level < 0 || p->feedback_level > 2 ||
      !(p->r_sample[2] > 0.0 && p->r_sample[2] < 1.0) || !(p->r_sample[0] > 0.0) ||
      !(p->r_sample[1] > 0.0))
    return IMAGO_ERR_INVALID;
  std::memcpy(c->rv, s->real_vectors, sizeof c->rv);
  recip_vectors(c);
  c->Tb = -std::log(s->basis_fn_convg);
  c->Te = -std::log(s->electro_convg);
  c->npt = s->num_pot_types;
  c->nps = s->num_pot_sites;
  int off = 0;
  c->min_pot_alpha = 10000.0;
  for (int t = 0; t < c->npt; ++t) {
    PType q{};
    q.n = s->pot_type_num_alphas[t];
    if (q.n < 1 || q.n > kMaxPotAlphas) return IMAGO_ERR_RANGE;
    q.off = off;
    q.z = s->pot_type_nuc_charge[t];
    q.nucalpha = s->pot_type_nuc_alpha[t];
    q.element = s->pot_type_element ? s->pot_type_element[t] : t + 1;
    q.covrad = p->covalent_radius[t];
    for (int a = 0; a < q.n; ++a) {
      const double x = s->pot_type_alphas[off + a];
      if (!(x > 0.0) || (a && !(x > s->pot_type_alphas[off + a - 1])))
        return IMAGO_ERR_INVALID;
      c->alpha.push_back(x);
    }
    c->min_pot_alpha = std::min(c->min_pot_alpha, c->alpha[off]);
    off += q.n;
    c->pt.push_back(q);
  }
  c->P = off;
  c->ps_type.resize(c->nps);
  c->ps_pos.assign(s->pot_site_pos, s->pot_site_pos + 3 * c->nps);
  for (int i = 0; i < c->nps; ++i) {
    const int t = s->pot_site_type[i] - 1;
    if (t < 0 || t >= c->npt || (i && t < c->ps_type[i - 1])) return IMAGO_ERR_INVALID;
    c->ps_type[i] = t;
    c->pt[t].mult++;
  }
  c->min_atom_alpha = 100.0;
  const int *noa = s->type_num_orb_alphas;
  int aoff = 0;
  for (int t = 0; t < s->num_atom_types; ++t) {
    c->min_atom_alpha = std::min(c->min_atom_alpha, s->type_alphas[aoff]);
    aoff += noa[4 * t];
  }
  c->xc = p->xc_code;
  c->feedback = p->feedback_level;
  c->relax = p->relax_factor;
  c->convg = p->convergence_test;
  c->nelec = p->num_electrons;
  return IMAGO_OK;
}

// initializeLattice (lattice.f90:330-444): both lists.
void make_lattices(imago_scf *c) {
  double lim = c->Tb * std::max(2.0 / c->min_atom_alpha,
                                1.0 / c->min_pot_alpha + 0.5 / c->min_atom_alpha);
  double maxsq = 0.0;
  for (int i = 0; i < 3; ++i) {
    double l2 = 0.0;
    for (int x = 0; x < 3; ++x) l2 += c->rv[3 * i + x] * c->rv[3 * i + x];
    maxsq = std::max(l2, maxsq);
  }
  lim = lim + 0.75 * maxsq + std::sqrt(3.0 * maxsq * lim);
  lim = std::max(lim, 2.0 * c->Tb / c->min_atom_alpha);
  lattice_points(c->rv, lim, c->cells, c->csize);
  lattice_points(c->recip, 4.0 * c->Te * c->min_pot_alpha, c->rcells, c->rcsize);
}

// initPotStructures' integration constants (potential.f90:149-160):
// multiplicity * (pi / alpha)^(3/2), as pi^(3/2) / alpha^(3/2).
void make_intg(imago_scf *c) {
  c->intg.assign(c->P, 0.0);
  const double pi32 = std::pow(kPi, 1.5);
  for (const PType &t : c->pt)
    for (int a = 0; a < t.n; ++a)
      c->intg[t.off + a] = (double)t.mult * pi32 / std::pow(c->alpha[t.off + a], 1.5);
}

// makeCoreRho (coreCharge.f90:27-578): per potential type with core states
// (the type index shared with the atom types), the core density's
// projections onto the type's Gaussians, fitted with the Gaussians' self
// overlap, scaled to the core electron count and corrected by a Lagrange
// multiplier on the charge.
int make_core_rho(imago_scf *c, const imago_system *s) {
  c->core_rho.assign(c->P, 0.0);
  const double pi32 = std::pow(kPi, 1.5);
  double factor[4];
  const double num[4] = {1.0, 3.0, 15.0, 105.0}, den[4] = {4.0, 8.0, 16.0, 32.0};
  for (int k = 0; k < 4; ++k)
    factor[k] = std::sqrt(kPi) * num[k] / den[k] * (2 * k + 1) * 2.0 * 2.0;
  int aoff = 0, foff = 0, coff = 0;
  std::vector<int> type_aoff(s->num_atom_types), type_foff(s->num_atom_types),
      type_coff(s->num_atom_types);
  for (int t = 0; t < s->num_atom_types; ++t) {
    type_aoff[t] = aoff;
    type_foff[t] = foff;
    type_coff[t] = coff;
    aoff += s->type_num_orb_alphas[4 * t];
    const int nf = s->type_num_core_fns[t] + s->type_num_vale_fns[t];
    for (int f = 0; f < nf; ++f) coff += s->type_num_orb_alphas[4 * t + s->fn_l[foff + f]];
    foff += nf;
  }
  std::vector<bool> first(c->npt, false);
  for (int i = 0; i < c->nps; ++i)
    if (i == 0 || c->ps_type[i] != c->ps_type[i - 1]) first[c->ps_type[i]] = true;
  for (int t = 0; t < c->npt; ++t) {
    if (!first[t] || t >= s->num_atom_types) continue;
    const int ncore = s->type_num_core_fns[t];
    if (ncore == 0) continue;
    const int *noa = s->type_num_orb_alphas + 4 * t;
    const double *aa = s->type_alphas + type_aoff[t];
    const int np = c->pt[t].n;
    const double *pa = &c->alpha[c->pt[t].off];
    int maxl = 0, nstates = 0;
    std::vector<int> cl(ncore);
    std::vector<const double *> cc(ncore);
    int co = type_coff[t];
    for (int f = 0; f < ncore; ++f) {
      cl[f] = s->fn_l[type_foff[t] + f];
      cc[f] = s->fn_coeffs + co;
      co += noa[cl[f]];
      maxl = std::max(maxl, cl[f]);
      nstates += 2 * cl[f] + 1;
    }
    std::vector<double> ov(2 * np), ints(np), self((size_t)np * np);
    const int na = noa[0];
    std::vector<double> af((size_t)na * na * 4, 0.0);
    for (int j = 0; j < np; ++j) {
      double o1 = 0.0;
      ov[np + j] = pi32 / std::pow(pa[j], 1.5);
      ints[j] = ov[np + j];
      for (int k = 0; k <= maxl; ++k)
        for (int l = 0; l < noa[k]; ++l)
          for (int m = l; m < noa[k]; ++m) {
            const double range = 1.0 / (pa[j] + aa[l] + aa[m]);
            double pw = 1.0;
            for (int e = 0; e <= k; ++e) pw *= range;
            af[((size_t)k * na + l) * na + m] = factor[k] * std::sqrt(range) * pw;
          }
      for (int f = 0; f < ncore; ++f) {
        const int k = cl[f];
        const double *cf = cc[f];
        for (int l = 0; l < noa[k]; ++l) {
          for (int m = l; m < noa[k]; ++m)
            o1 = o1 + af[((size_t)k * na + l) * na + m] * cf[l] * cf[m];
          o1 = o1 - af[((size_t)k * na + l) * na + l] * cf[l] * cf[l] * 0.5;
        }
      }
      ov[j] = o1;
      for (int k = j; k < np; ++k) {
        self[(size_t)k * np + j] = pi32 / std::pow(pa[j] + pa[k], 1.5);
        self[(size_t)j * np + k] = self[(size_t)k * np + j];
      }
    }
    int rc = solve_spd(np, 2, self.data(), ov.data());
    if (rc) return rc;
    const double ne = 2.0 * nstates;
    const double delta = (ne - seq_dot(ov.data(), ints.data(), np)) /
                         seq_dot(ov.data() + np, ints.data(), np);
    for (int j = 0; j < np; ++j) c->core_rho[c->pt[t].off + j] = ov[j] + delta * ov[np + j];
  }
  return IMAGO_OK;
}

// getECMeshParameters + the ray walk of makeECMeshAndOverlap
// (exchCorr.f90:63-342, 440-600): sample directions (makeSampleVectors,
// exchCorr.f90:920-980), per site and direction the largest radius before
// the bisecting planes towards the neighbours (weighted by the covalent
// radii), then points from that radius inward by the spacing factor with
// their radial weights.
void make_mesh_points(imago_scf *c, const imago_scf_params *p) {
  const int nv = p->num_sample_vectors;
  std::vector<double> vec(3 * nv);
  {
    std::vector<double> h(nv), th(nv), ph(nv);
    h[0] = -1.0;
    h[nv - 1] = 1.0;
    for (int k = 1; k < nv - 1; ++k) h[k] = -1.0 + 2.0 * ((k + 1) - 1.0) / (nv - 1.0);
    for (int k = 0; k < nv; ++k) th[k] = std::acos(h[k]);
    ph[0] = 0.0;
    ph[nv - 1] = 0.0;
    for (int k = 1; k < nv - 1; ++k) {
      ph[k] = ph[k - 1] + 3.6 / std::sqrt((double)nv) * 1.0 / std::sqrt(1.0 - h[k] * h[k]);
      while (ph[k] > 2.0 * kPi) ph[k] = ph[k] - 2.0 * kPi;
    }
    for (int k = 0; k < nv; ++k) {
      vec[3 * k] = std::sin(th[k]) * std::cos(ph[k]);
      vec[3 * k + 1] = std::sin(th[k]) * std::sin(ph[k]);
      vec[3 * k + 2] = std::cos(th[k]);
    }
  }
  const int nreps = std::min(64, (int)c->csize.size());
  const int ns = c->nps;
  std::vector<double> lsep(3 * ns, 0.0), list((size_t)3 * nreps * ns, 0.0);
  auto live = [&](int i) { return !(c->pt[c->ps_type[i]].covrad < kSmallThresh); };
  for (int i = 0; i < ns; ++i) {
    if (!live(i)) continue;
    double L[3];
    nearest_vec(c->rv, c->inv, &c->ps_pos[3 * i], L);
    for (int x = 0; x < 3; ++x) lsep[3 * i + x] = c->ps_pos[3 * i + x] - L[x];
    for (int j = 0; j < nreps; ++j)
      for (int x = 0; x < 3; ++x)
        list[((size_t)i * nreps + j) * 3 + x] = lsep[3 * i + x] + c->cells[3 * j + x];
  }
  const double max_r = std::sqrt(p->r_sample[1] / c->min_pot_alpha);
  std::vector<double> rmax((size_t)ns * nv, 0.0);
  auto radii = [&](int i0, int i1) {
    for (int i = i0; i < i1; ++i) {
      if (!live(i)) continue;
      const double cri = c->pt[c->ps_type[i]].covrad;
      for (int j = 0; j < nv; ++j) {
        double cur = max_r;
        for (int k = 0; k < ns; ++k) {
          if (!live(k)) continue;
          const double f = cri / (cri + c->pt[c->ps_type[k]].covrad);
          for (int l = 0; l < nreps; ++l) {
            double sep[3];
            for (int x = 0; x < 3; ++x)
              sep[x] = f * (list[((size_t)k * nreps + l) * 3 + x] - list[(size_t)i * nreps * 3 + x]);
            const double dot = sep[0] * vec[3 * j] + sep[1] * vec[3 * j + 1] + sep[2] * vec[3 * j + 2];
            if (dot <= kSmallThresh) continue;
            cur = std::min((sep[0] * sep[0] + sep[1] * sep[1] + sep[2] * sep[2]) / dot, cur);
          }
        }
        rmax[(size_t)i * nv + j] = cur;
      }
    }
  };
  const int nth = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  std::vector<std::thread> th;
  const int per = (ns + nth - 1) / nth;
  for (int q = 0; q < nth; ++q) {
    const int i0 = q * per, i1 = std::min(ns, i0 + per);
    if (i0 < i1) th.emplace_back(radii, i0, i1);
  }
  for (auto &t : th) t.join();
  const double space = p->r_sample[2], space_sqrt = std::sqrt(space);
  const double wf = (1.0 - space) / space_sqrt;
  const double *wt = p->ang_weights;
  c->site_n.assign(ns, 0);
  c->site_off.assign(ns, 0);
  c->pts.clear();
  c->w.clear();
  for (int i = 0; i < ns; ++i) {
    c->site_off[i] = (int)c->w.size();
    if (!live(i)) continue;
    const PType &t = c->pt[c->ps_type[i]];
    const double half = t.covrad / 2.0;
    const double minr = std::sqrt(p->r_sample[0] / c->alpha[t.off + t.n - 1]);
    for (int j = 0; j < nv; ++j) {
      double r = rmax[(size_t)i * nv + j];
      int wi = 1;
      double endf = 0.5;
      const double *v = &vec[3 * j];
      while (true) {
        for (int x = 0; x < 3; ++x) c->pts.push_back(r * v[x] + lsep[3 * i + x]);
        c->w.push_back(wt[wi] * wf * endf * (r * r * r));
        endf = 1.0;
        if (r < half || r < minr) wi = 0;
        if (wt[wi] < kSmallThresh) break;
        if (r < minr) {
          r = r * space_sqrt;
          for (int x = 0; x < 3; ++x) c->pts.push_back(0.75 * r * v[x] + lsep[3 * i + x]);
          c->w.push_back(wt[0] * (r * r * r) / 3.0);
          break;
        }
        r = r * space;
      }
    }
    c->site_n[i] = (int)c->w.size() - c->site_off[i];
  }
  c->npoints = (int)c->w.size();
}

// recipCellExp and minReducedAlphaSqrt of residualQ (elecStat.f90:858-889):
// recomputed at the first site of a type whose element differs from the
// previous type's, so a type that follows one of the same element reuses
// its table.
void residual_tables(const imago_scf *c, std::vector<int> &table_of_type,
                     std::vector<double> &rce, std::vector<double> &mra) {
  table_of_type.assign(c->npt, 0);
  std::vector<int> owner;
  int last_el = 0, cur = -1;
  for (int t = 0; t < c->npt; ++t) {
    if (c->pt[t].element != last_el) {
      owner.push_back(t);
      cur = (int)owner.size() - 1;
    }
    last_el = c->pt[t].element;
    table_of_type[t] = cur;
  }
  const int ng = (int)c->rcsize.size();
  rce.assign((size_t)owner.size() * ng * kMaxPotAlphas, 0.0);
  mra.assign(owner.size() * kMaxPotAlphas, 0.0);
  for (size_t q = 0; q < owner.size(); ++q) {
    const PType &t = c->pt[owner[q]];
    for (int j = 0; j < t.n; ++j) {
      const double a = c->alpha[t.off + j];
      const double mu = a * c->min_pot_alpha / (a + c->min_pot_alpha);
      mra[q * kMaxPotAlphas + j] = std::sqrt(mu);
      const double inv4 = 0.25 / mu;
      for (int g = 1; g < ng; ++g)
        rce[((size_t)q * ng + g) * kMaxPotAlphas + j] =
            std::exp(-c->rcsize[g] * inv4) / c->rcsize[g];
    }
  }
}

int electrostatics(imago_scf *c) {
  const int ns = c->nps, P = c->P;
  const long long npairs = (long long)ns * ns;
  std::vector<double> minsep(3 * npairs);
  for (int i = 0; i < ns; ++i)
    for (int j = 0; j < ns; ++j) {
      double v[3], L[3];
      for (int x = 0; x < 3; ++x) v[x] = c->ps_pos[3 * i + x] - c->ps_pos[3 * j + x];
      nearest_vec(c->rv, c->inv, v, L);
      for (int x = 0; x < 3; ++x) minsep[3 * ((long long)i * ns + j) + x] = v[x] - L[x];
    }
  std::vector<int> tab;
  std::vector<double> rce, mra;
  residual_tables(c, tab, rce, mra);
  const double *d_minsep, *d_rce, *d_mra;
  const int *d_tab;
  int rc = upload(c, minsep, &d_minsep);
  if (!rc) rc = upload(c, rce, &d_rce);
  if (!rc) rc = upload(c, mra, &d_mra);
  if (!rc) rc = upload(c, tab, &d_tab);
  if (rc) return rc;
  const long long stride = 3 * kMaxPotAlphas * kMaxPotAlphas + kMaxPotAlphas;
  double *part, *rpart, *outm;
  if ((rc = dalloc(c, &part, (size_t)(npairs * stride)))) return rc;
  if ((rc = dalloc(c, &rpart, (size_t)(npairs * kMaxPotAlphas)))) return rc;
  const size_t nout = (size_t)3 * P * P + P + (size_t)c->npt * P;
  if ((rc = dalloc(c, &outm, nout))) return rc;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, c->stream);
  k_es_pairs<<<(unsigned)npairs, kEsThreads, 0, c->stream>>>(c->dev, d_minsep, stride, part);
  k_res_pairs<<<(unsigned)npairs, kResThreads, 0, c->stream>>>(
      c->dev, d_minsep, d_tab, d_rce, d_mra, c->min_pot_alpha, c->volume, rpart);
  const long long nthr = (long long)P * P + P + (long long)c->npt * P;
  k_es_reduce<<<(unsigned)((nthr + 127) / 128), 128, 0, c->stream>>>(
      c->dev, part, stride, rpart, outm, outm + (size_t)P * P, outm + 2 * (size_t)P * P,
      outm + 3 * (size_t)P * P, outm + 3 * (size_t)P * P + P, c->npt);
  cudaEventRecord(e1, c->stream);
  std::vector<double> h(nout);
  IMAGO_CUDA(cudaMemcpyAsync(h.data(), outm, nout * sizeof(double), cudaMemcpyDeviceToHost,
                             c->stream));
  IMAGO_CUDA(cudaStreamSynchronize(c->stream));
  IMAGO_CUDA(cudaGetLastError());
  cudaEventElapsedTime(&c->ms[0], e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  const size_t PP = (size_t)P * P;
  c->nl_neut.assign(h.begin(), h.begin() + PP);
  c->l_neut.assign(h.begin() + PP, h.begin() + 2 * PP);
  c->pot_ol.assign(h.begin() + 2 * PP, h.begin() + 3 * PP);
  c->nl_nuc.assign(h.begin() + 3 * PP, h.begin() + 3 * PP + P);
  c->nl_res.assign(h.begin() + 3 * PP + P, h.end());
  // the local nuclear term (elecStat.f90:509-515): a site with itself
  c->l_nuc.assign(P, 0.0);
  for (int i = 0; i < ns; ++i)
    for (int j = 0; j < ns; ++j) {
      double d2 = 0.0;
      for (int x = 0; x < 3; ++x) {
        const double d = c->ps_pos[3 * i + x] - c->ps_pos[3 * j + x];
        d2 += d * d;
      }
      if (d2 < kSmallThresh) {
        const PType &t = c->pt[c->ps_type[i]];
        for (int a = 0; a < t.n; ++a)
          c->l_nuc[t.off + a] = c->l_nuc[t.off + a] - 2.0 * kPi * t.z / c->alpha[t.off + a];
      }
    }
  return IMAGO_OK;
}

int mesh_operator(imago_scf *c) {
  const int P = c->P, np = c->npoints;
  const double *d_pts;
  int rc = upload(c, c->pts, &d_pts);
  if (rc) return rc;
  if ((rc = dalloc(c, &c->d_op, (size_t)np * P))) return rc;
  const double *dw;
  if ((rc = upload(c, c->w, &dw))) return rc;
  c->d_w = const_cast<double *>(dw);
  std::vector<int> so(2 * c->nps);
  for (int i = 0; i < c->nps; ++i) {
    so[i] = c->site_off[i];
    so[c->nps + i] = c->site_n[i];
  }
  const int *dso;
  if ((rc = upload(c, so, &dso))) return rc;
  c->d_site = const_cast<int *>(dso);
  const int nchunk = std::max(1, (np + kChunkPoints - 1) / kChunkPoints);
  const int nval = P * (P + 1) / 2;
  c->buf_doubles = (size_t)nchunk * std::max(nval, 3 * P) + 3 * (size_t)np + 8 * P +
                   2 * (size_t)c->nps + (size_t)nval;
  if ((rc = dalloc(c, &c->d_buf, c->buf_doubles))) return rc;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, c->stream);
  if (np) {
    const long long nthr = (long long)np * c->npt;
    k_xc_operator<<<(unsigned)((nthr + 127) / 128), 128, 0, c->stream>>>(c->dev, d_pts, np,
                                                                       c->npt, c->d_op);
    k_xc_chunks<<<nchunk, 256, 0, c->stream>>>(c->d_op, c->d_w, nullptr, np, P, 0, c->d_buf);
  }
  double *ovl = c->d_buf + (size_t)nchunk * std::max(nval, 3 * P);
  if (np)
    k_reduce_chunks<<<(nval + 127) / 128, 128, 0, c->stream>>>(c->d_buf, nchunk, nval, ovl);
  else
    IMAGO_CUDA(cudaMemsetAsync(ovl, 0, nval * sizeof(double), c->stream));
  cudaEventRecord(e1, c->stream);
  std::vector<double> h(nval);
  IMAGO_CUDA(cudaMemcpyAsync(h.data(), ovl, nval * sizeof(double), cudaMemcpyDeviceToHost,
                             c->stream));
  IMAGO_CUDA(cudaStreamSynchronize(c->stream));
  IMAGO_CUDA(cudaGetLastError());
  cudaEventElapsedTime(&c->ms[1], e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->xc_ol.assign((size_t)P * P, 0.0);
  for (int k = 0; k < P; ++k)
    for (int a = 0; a <= k; ++a) c->xc_ol[(size_t)k * P + a] = h[k * (k + 1) / 2 + a];
  return IMAGO_OK;
}

}  // namespace

extern "C" {

int imago_scf_create(const imago_system *sys, const imago_scf_params *params, int device,
                     void *stream, imago_scf **out) {
  if (!out) return IMAGO_ERR_INVALID;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return IMAGO_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= ndev) return IMAGO_ERR_INVALID;
  std::unique_ptr<imago_scf> c(new imago_scf());
  int rc = read_system(c.get(), sys, params);
  if (rc) return rc;
  c->device = device;
  IMAGO_CUDA(cudaSetDevice(device));
  if (stream) {
    c->stream = static_cast<cudaStream_t>(stream);
  } else {
    IMAGO_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    c->own_stream = true;
  }
  make_lattices(c.get());
  make_intg(c.get());
  if ((rc = make_core_rho(c.get(), sys))) {
    imago_scf_destroy(c.release());
    return rc;
  }
  make_mesh_points(c.get(), params);
  // device tables
  ScfDev &d = c->dev;
  d.nps = c->nps;
  d.npt = c->npt;
  d.pot_dim = c->P;
  d.Te = c->Te;
  std::memcpy(d.rv, c->rv, sizeof d.rv);
  std::memcpy(d.inv, c->inv, sizeof d.inv);
  std::vector<int> off(c->npt), num(c->npt);
  std::vector<double> z(c->npt), nuc(c->npt);
  for (int t = 0; t < c->npt; ++t) {
    off[t] = c->pt[t].off;
    num[t] = c->pt[t].n;
    z[t] = c->pt[t].z;
    nuc[t] = c->pt[t].nucalpha;
  }
  d.ncell = (int)c->csize.size();
  d.nrecip = (int)c->rcsize.size();
  if ((rc = upload(c.get(), c->ps_type, &d.ps_type)) ||
      (rc = upload(c.get(), c->ps_pos, &d.ps_pos)) || (rc = upload(c.get(), off, &d.pt_off)) ||
      (rc = upload(c.get(), num, &d.pt_n)) || (rc = upload(c.get(), z, &d.pt_z)) ||
      (rc = upload(c.get(), nuc, &d.pt_nuc)) || (rc = upload(c.get(), c->alpha, &d.alpha)) ||
      (rc = upload(c.get(), c->cells, &d.cell)) || (rc = upload(c.get(), c->csize, &d.csize)) ||
      (rc = upload(c.get(), c->rcells, &d.rcell)) || (rc = electrostatics(c.get())) ||
      (rc = mesh_operator(c.get()))) {
    imago_scf_destroy(c.release());
    return rc;
  }
  *out = c.release();
  return IMAGO_OK;
}

void imago_scf_destroy(imago_scf *c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (void *p : c->allocs) cudaFree(p);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  cudaGetLastError();
  delete c;
}

int imago_scf_get_dims(const imago_scf *c, imago_scf_dims *d) {
  if (!c || !d) return IMAGO_ERR_INVALID;
  d->pot_dim = c->P;
  d->num_pot_types = c->npt;
  d->num_pot_sites = c->nps;
  d->num_cells_real = (int)c->csize.size();
  d->num_cells_recip = (int)c->rcsize.size();
  d->num_mesh_points = c->npoints;
  return IMAGO_OK;
}

int imago_scf_setup_arrays(const imago_scf *c, double *pot_ol, double *nl_neut,
                           double *l_neut, double *nl_nuc, double *l_nuc, double *nl_res,
                           double *core, double *xc_ol, double *intg) {
  if (!c) return IMAGO_ERR_INVALID;
  auto cp = [](const std::vector<double> &v, double *o) {
    if (o) std::copy(v.begin(), v.end(), o);
  };
  cp(c->pot_ol, pot_ol);
  cp(c->nl_neut, nl_neut);
  cp(c->l_neut, l_neut);
  cp(c->nl_nuc, nl_nuc);
  cp(c->l_nuc, l_nuc);
  cp(c->nl_res, nl_res);
  cp(c->core_rho, core);
  cp(c->xc_ol, xc_ol);
  cp(c->intg, intg);
  return IMAGO_OK;
}

int imago_scf_mesh(const imago_scf *c, int *site_points, double *radial_weight,
                   double *op) {
  if (!c) return IMAGO_ERR_INVALID;
  if (site_points) std::copy(c->site_n.begin(), c->site_n.end(), site_points);
  if (radial_weight) std::copy(c->w.begin(), c->w.end(), radial_weight);
  if (op && c->npoints) {
    IMAGO_CUDA(cudaSetDevice(c->device));
    IMAGO_CUDA(cudaMemcpyAsync(op, c->d_op, (size_t)c->npoints * c->P * sizeof(double),
                               cudaMemcpyDeviceToHost, c->stream));
    IMAGO_CUDA(cudaStreamSynchronize(c->stream));
  }
  return IMAGO_OK;
}

int imago_scf_lattice(const imago_scf *c, double *rd, double *rs, double *gd, double *gs) {
  if (!c) return IMAGO_ERR_INVALID;
  if (rd) std::copy(c->cells.begin(), c->cells.end(), rd);
  if (rs) std::copy(c->csize.begin(), c->csize.end(), rs);
  if (gd) std::copy(c->rcells.begin(), c->rcells.end(), gd);
  if (gs) std::copy(c->rcsize.begin(), c->rcsize.end(), gs);
  return IMAGO_OK;
}

int imago_scf_reset_history(imago_scf *c) {
  if (!c) return IMAGO_ERR_INVALID;
  c->hist = false;
  c->iter = 1;
  return IMAGO_OK;
}

int imago_scf_timings(const imago_scf *c, double ms[3]) {
  if (!c || !ms) return IMAGO_ERR_INVALID;
  for (int i = 0; i < 3; ++i) ms[i] = c->ms[i];
  return IMAGO_OK;
}

// makeSCFPot (potentialUpdate.F90:53-1866) for spin 1, rel 0.
int imago_scf_pot_update(imago_scf *c, const double *pot_rho, double nuc_trace,
                         double kin_trace, double *coeffs, double *result) {
  if (!c || !pot_rho || !coeffs || !result) return IMAGO_ERR_INVALID;
  const int P = c->P;
  IMAGO_CUDA(cudaSetDevice(c->device));
  // generalRho(:, 1..7), column-major
  std::vector<double> gr((size_t)P * 8, 0.0);
  auto G = [&](int i, int col) -> double & { return gr[(size_t)(col - 1) * P + i]; };
  for (int i = 0; i < P; ++i) {
    G(i, 1) = pot_rho[i];
    G(i, 2) = c->intg[i];
  }
  int rc = solve_spd(P, 2, c->pot_ol.data(), gr.data());
  if (rc) return rc;
  const double fitted = seq_dot(c->intg.data(), &G(0, 1), P);
  const double ediff = c->nelec - fitted;
  {
    double den = 0.0;
    for (int i = 0; i < P; ++i) den = den + c->intg[i] * G(i, 2);
    for (int i = 0; i < P; ++i) G(i, 2) = G(i, 1) + G(i, 2) * ediff / den;
  }
  for (int i = 0; i < P; ++i) {
    G(i, 3) = c->core_rho[i];
    G(i, 1) = G(i, 2) + G(i, 3);
    G(i, 4) = G(i, 1);
    G(i, 5) = G(i, 6) = G(i, 7) = 0.0;
  }
  for (int t = 0; t < c->npt; ++t) {
    const PType &q = c->pt[t];
    const double zc = q.z * q.mult;
    const int b = q.off, e = q.off + q.n - 1;
    double sum = 0.0;
    for (int i = b; i <= e; ++i) sum = sum + c->intg[i] * G(i, 1);
    G(b, 5) = (sum - zc) / c->intg[b];
    G(b, 4) = G(b, 1) - G(b, 5);
    G(t, 6) = G(b, 5);
    G(e, 7) = -zc / c->intg[e];
  }
  // elecStatPot(:, 1..6)
  std::vector<double> es((size_t)P * 6, 0.0);
  auto E = [&](int i, int col) -> double & { return es[(size_t)(col - 1) * P + i]; };
  std::vector<double> vneut(P);
  for (int i = 0; i < P; ++i) vneut[i] = G(i, 2) - G(i, 5);
  for (int i = 0; i < P; ++i) {
    E(i, 1) = seq_dot(&c->nl_neut[(size_t)i * P], &G(0, 4), P);
    E(i, 2) = seq_dot(&c->l_neut[(size_t)i * P], vneut.data(), P);
    E(i, 3) = seq_dot(&c->l_neut[(size_t)i * P], &G(0, 3), P);
    E(i, 4) = c->nl_nuc[i];
    E(i, 5) = c->l_nuc[i];
    E(i, 6) = seq_dot(&c->nl_res[(size_t)i * c->npt], &G(0, 6), c->npt);
  }
  double es_energy = 0.0;
  for (int i = 0; i < P; ++i)
    es_energy = es_energy + (0.5 * (G(i, 1) + G(i, 7)) * (E(i, 1) + E(i, 6)) +
                             0.5 * G(i, 2) * (E(i, 2) + E(i, 3) + E(i, 5)) +
                             0.5 * (G(i, 2) - G(i, 5)) * (E(i, 3) + E(i, 5)));
  {
    double s = 0.0;
    for (int i = 0; i < P; ++i) s = s + G(i, 2) * E(i, 4);
    es_energy = es_energy - s + nuc_trace;
  }
  for (int i = 0; i < P; ++i) {
    E(i, 1) = E(i, 1) + E(i, 2) + E(i, 3) - E(i, 4) + E(i, 5);
    E(i, 2) = E(i, 6);
  }
  if ((rc = solve_spd(P, 2, c->pot_ol.data(), es.data()))) return rc;
  // exchange-correlation on the mesh
  const int np = c->npoints;
  const int nchunk = std::max(1, (np + kChunkPoints - 1) / kChunkPoints);
  double *part = c->d_buf;
  double *g = part + (size_t)nchunk * std::max(P * (P + 1) / 2, 3 * P);
  double *dr = g + 3 * (size_t)np;  // [P] total, [P] core, [3P] result, [P] dv, [2 nps]
  double *dres = dr + 2 * P, *ddv = dres + 3 * P, *ddelta = ddv + P;
  std::vector<double> rho2(2 * (size_t)P);
  for (int i = 0; i < P; ++i) {
    rho2[i] = G(i, 1);
    rho2[P + i] = G(i, 3);
  }
  std::vector<double> xcp(3 * (size_t)P, 0.0);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, c->stream);
  IMAGO_CUDA(cudaMemcpyAsync(dr, rho2.data(), 2 * P * sizeof(double), cudaMemcpyHostToDevice,
                             c->stream));
  if (np) {
    k_xc_points<<<(np + 7) / 8, 256, 0, c->stream>>>(c->d_op, c->d_w, dr, dr + P, np, P, c->xc,
                                                     g);
    k_xc_chunks<<<nchunk, 128, 0, c->stream>>>(c->d_op, c->d_w, g, np, P, 1, part);
    k_reduce_chunks<<<(3 * P + 127) / 128, 128, 0, c->stream>>>(part, nchunk, 3 * P, dres);
    IMAGO_CUDA(cudaMemcpyAsync(xcp.data(), dres, 3 * P * sizeof(double),
                               cudaMemcpyDeviceToHost, c->stream));
  }
  IMAGO_CUDA(cudaStreamSynchronize(c->stream));
  IMAGO_CUDA(cudaGetLastError());
  if ((rc = solve_spd(P, 3, c->xc_ol.data(), xcp.data()))) return rc;
  double xc_energy = 0.0;
  for (int i = 0; i < P; ++i)
    xc_energy = xc_energy + seq_dot(&c->pot_ol[(size_t)i * P], &xcp[P], P) * G(i, 1) -
                seq_dot(&c->pot_ol[(size_t)i * P], &xcp[2 * P], P) * G(i, 3);
  const double total = kin_trace + es_energy + xc_energy;
  result[0] = total;
  result[1] = kin_trace;
  result[2] = es_energy;
  result[3] = xc_energy;
  result[4] = ediff;
  if (total > 0.0) return IMAGO_ERR_SCF;
  // Anderson mixing (potentialUpdate.F90:1303-1321, 1620-1680)
  std::vector<double> xl0(coeffs, coeffs + P), yl0(P), out(P);
  for (int i = 0; i < P; ++i) yl0[i] = E(i, 1) + E(i, 2) + xcp[i];
  if (!c->hist) {
    c->xl1 = c->xl2 = xl0;
    c->yl1 = c->yl2 = yl0;
    c->hist = true;
  }
  for (int i = 0; i < P; ++i) out[i] = yl0[i] - xl0[i];
  // real-space convergence measure
  double delta = 0.0;
  if (np) {
    std::vector<double> dd(2 * (size_t)c->nps);
    IMAGO_CUDA(cudaMemcpyAsync(ddv, out.data(), P * sizeof(double), cudaMemcpyHostToDevice,
                               c->stream));
    k_xc_delta<<<c->nps, 256, 0, c->stream>>>(c->d_op, c->d_w, c->d_site, c->d_site + c->nps,
                                             ddv, P, ddelta);
    cudaEventRecord(e1, c->stream);
    IMAGO_CUDA(cudaMemcpyAsync(dd.data(), ddelta, dd.size() * sizeof(double),
                               cudaMemcpyDeviceToHost, c->stream));
    IMAGO_CUDA(cudaStreamSynchronize(c->stream));
    IMAGO_CUDA(cudaGetLastError());
    cudaEventElapsedTime(&c->ms[2], e0, e1);
    for (int i = 0; i < c->nps; ++i) {
      if (c->site_n[i] == 0) continue;
      delta = std::max(std::sqrt(dd[2 * i] / dd[2 * i + 1]), delta);
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  double th1 = 0.0, th2 = 0.0;
  if (c->feedback != 0 && c->iter > 1) {
    std::vector<double> r0(P), r1(P), r2(P), d1(P), d2(P);
    for (int i = 0; i < P; ++i) {
      r0[i] = yl0[i] - xl0[i];
      r1[i] = c->yl1[i] - c->xl1[i];
      r2[i] = c->yl2[i] - c->xl2[i];
      d1[i] = r0[i] - r1[i];
      d2[i] = r0[i] - r2[i];
    }
    double s11 = 0.0, s12 = 0.0, s22 = 0.0, t1 = 0.0, t2 = 0.0;
    for (int j = 0; j < P; ++j) {
      double a = 0.0, b = 0.0;
      for (int i = 0; i < P; ++i) {
        const double x = c->pot_ol[(size_t)j * P + i] * d1[j];
        a = a + x * d1[i];
        b = b + x * r0[i];
      }
      s11 = s11 + a;
      t1 = t1 + b;
    }
    for (int j = 0; j < P; ++j) {
      double a = 0.0, b = 0.0, d = 0.0;
      for (int i = 0; i < P; ++i) {
        const double x = c->pot_ol[(size_t)j * P + i] * d2[j];
        a = a + x * d1[i];
        b = b + x * d2[i];
        d = d + x * r0[i];
      }
      s12 = s12 + a;
      s22 = s22 + b;
      t2 = t2 + d;
    }
    th1 = t1 / s11;
    if (c->feedback != 1 && c->iter > 2) {
      const double det = s11 * s22 - s12 * s12;
      if (det / (s11 * s22) >= 0.01) {
        th1 = (s22 * t1 - s12 * t2) / det;
        th2 = (-s12 * t1 + s11 * t2) / det;
      }
    }
  }
  for (int i = 0; i < P; ++i)
    coeffs[i] = (1.0 - c->relax) *
                    ((1.0 - th1 - th2) * xl0[i] + th1 * c->xl1[i] + th2 * c->xl2[i]) +
                c->relax * ((1.0 - th1 - th2) * yl0[i] + th1 * c->yl1[i] + th2 * c->yl2[i]);
  c->xl2 = c->xl1;
  c->xl1 = xl0;
  c->yl2 = c->yl1;
  c->yl1 = yl0;
  int converged = 0;
  if (delta < c->convg)
    converged = 1;
  else
    c->iter = c->iter + 1;
  result[5] = delta;
  result[6] = converged;
  result[7] = c->iter;
  return IMAGO_OK;
}

}  // extern "C"
