// prim.cuh -- FP64 primitive integrals per shell-pair class on the device.
//
// A "class" (LA, LB) is the pair of lmAlphaIndex classes of the two
// primitives (basis.f90:138-146): all real solid harmonics up to l on each
// side, nsh = 1, 4, 9, 16.  Results are the reference's sh(16,16) blocks
// (gaussIntegrals.f90) restricted to nsh(LA) x nsh(LB), row-major.
//
//  * two-centre overlap and kinetic (overlap2CIntg, kinetic2CIntg): the
//    Obara-Saika recursions in separable 1D form;
//  * mass velocity (massvel2CIntg): <nabla^2 a|nabla^2 b> from the same
//    1D overlap tables, two orders higher;
//  * momentum and dipole (momentum2CIntg, dipole3CIntg): three Cartesian
//    components, the operator moved into one 1D factor;
//  * three-centre overlap and nuclear (electron3CIntg, nuclear3CIntg):
//    McMurchie-Davidson.  The product of the two orbital primitives is
//    expanded in Hermite Gaussians about P with coefficients E_t (they
//    depend only on the shell pair), so the lattice sum over potential
//    sites C accumulates only Hermite integrals Q_tuv(P - C), t+u+v <= LA+LB
//    (35 values for d-d), and the E transform runs once per shell pair and
//    term after the sum.
//  * The Boys function follows the reference's own branches
//    (gaussIntegrals.f90:16080-16221) so nuclear integrals agree with it.
#pragma once

#include "common.cuh"

namespace imago {

// ---------------------------------------------------------------- Boys --
// For T <= 0.1f the reference sums seven series terms with Gamma(n+1/2)
// written as default-REAL (single precision) literals; above it the closed
// forms in erf(sqrt T) and exp(-T).  Integer powers are formed as gfortran
// forms them (T^3 = T^2 T, T^4 = T^2 T^2, T^5 = T^3 T^2, T^6 = T^3 T^3).
__device__ __forceinline__ float gamma_half_f(int n) {
  const float g[14] = {1.7724538509055161f, 0.88622692545275805f,
                       1.3293403881791370f, 3.3233509704478426f,
                       11.631728396567450f, 52.342777784553533f,
                       287.88527781504416f, 1871.2543057977896f,
                       14034.407293483402f, 119292.46199460901f,
                       1133278.3889487833f, 11899423.083962219f,
                       136843365.46556622f, 1710542068.3195722f};
  return g[n];
}

template <int NMAX>
__device__ __forceinline__ void boys_ref(double T, double F[NMAX + 1]) {
  const double exp_T = exp(-T);
  const double sqrt_pi = sqrt(kPi);
  if (T <= (double)0.1f) {
    const double T2 = T * T, T3 = T2 * T, T4 = T2 * T2;
    const double T5 = T3 * T2, T6 = T3 * T3;
#pragma unroll
    for (int N = 0; N <= NMAX; ++N) {
      double a[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) a[k] = (double)gamma_half_f(N + k);
      F[N] = 0.5 * exp_T * a[0] *
             ((1 / a[1]) + (T / a[2]) + (T2 / a[3]) + (T3 / a[4]) +
              (T4 / a[5]) + (T5 / a[6]) + (T6 / a[7]));
    }
    return;
  }
  const double erf_T = erf(sqrt(T));
  F[0] = 0.5 * ((sqrt_pi / pow(T, 0.5)) * erf_T);
  const double T2 = T * T, T3 = T2 * T;
  const double Tp[7] = {1.0, T, T2, T3, T2 * T2, T3 * T2, T3 * T3};
  const double fact[13] = {1, 1, 2, 6, 24, 120, 720, 5040, 40320, 362880,
                           3628800, 39916800, 479001600};
  double c = 1.0, p4m = 1.0;
#pragma unroll
  for (int m = 1; m <= NMAX; ++m) {
    if (m > 1) c *= (double)(4 * m - 2);
    p4m *= 4.0;
    double erfterm = (sqrt_pi / (p4m * pow(T, (double)m + 0.5))) * erf_T;
    double s = 0.0, p4k = 1.0;
#pragma unroll
    for (int k = 1; k <= m; ++k) {
      const int r = m - k + 1;
      double den = (k == 1) ? fact[2 * r] * T : (p4k * fact[2 * r]) * Tp[k];
      double term = fact[r] / den;
      s = (k == 1) ? term : s + term;
      p4k *= 4.0;
    }
    double v = erfterm - exp_T * s;
    F[m] = (m == 1) ? v : c * v;
  }
}

// ------------------------------------------------------ 1D Obara-Saika --
// S[i][j] for a Gaussian product with exponent p, relative to the centres:
// S00 = 1, S_{i+1,j} = PA S_ij + (i S_{i-1,j} + j S_{i,j-1})/(2p), and the
// same with PB for j.
template <int IA, int JB>
__device__ __forceinline__ void os1d(double PA, double PB, double inv2p,
                                     double S[IA + 1][JB + 1]) {
  S[0][0] = 1.0;
#pragma unroll
  for (int i = 0; i < IA; ++i)
    S[i + 1][0] = PA * S[i][0] + (i > 0 ? i * inv2p * S[i - 1][0] : 0.0);
#pragma unroll
  for (int j = 0; j < JB; ++j)
#pragma unroll
    for (int i = 0; i <= IA; ++i) {
      double v = PB * S[i][j];
      if (i > 0) v += i * inv2p * S[i - 1][j];
      if (j > 0) v += j * inv2p * S[i][j - 1];
      S[i][j + 1] = v;
    }
}

// Write the real-solid-harmonic block from a Cartesian block
// pc[p * ncart(LB) + q].
template <int LA, int LB>
__device__ __forceinline__ void cart_to_sh(const double *pc, double *out) {
#pragma unroll
  for (int s1 = 0; s1 < nsh(LA); ++s1)
#pragma unroll
    for (int s2 = 0; s2 < nsh(LB); ++s2) {
      double v = 0.0;
#pragma unroll
      for (int k1 = 0; k1 < 3; ++k1) {
        if (k1 >= sh_nterm(s1)) break;
#pragma unroll
        for (int k2 = 0; k2 < 3; ++k2) {
          if (k2 >= sh_nterm(s2)) break;
          v += sh_coef(s1, k1) * sh_coef(s2, k2) *
               pc[sh_cart(s1, k1) * ncart(LB) + sh_cart(s2, k2)];
        }
      }
      out[s1 * nsh(LB) + s2] = v;
    }
}

// Two-centre overlap (KIN = false) or kinetic energy (KIN = true) between
// primitives a1 at A and a2 at B, written to out[nsh(LA) * nsh(LB)].
// Kinetic: the Obara-Saika kinetic recursion in separable form,
//   T00 = xi (1 - 2 xi X^2),
//   T_{i+1,j} = PA T_ij + (i T_{i-1,j} + j T_{i,j-1})/(2p)
//               + 2 xi (S_{i+1,j} - i/(2 a1) S_{i-1,j})   (and j likewise),
//   KE = pref (Tx Sy Sz + Sx Ty Sz + Sx Sy Tz).
template <int LA, int LB, bool KIN>
__device__ void prim2c(double a1, double a2, const double *A, const double *B,
                       double *out) {
  const double zeta = a1 + a2, xi = a1 * a2 / zeta, inv2p = 1.0 / (2.0 * zeta);
  double S[3][LA + 1][LB + 1];
  double T[3][LA + 1][LB + 1];
  double d2 = 0.0;
#pragma unroll
  for (int x = 0; x < 3; ++x) {
    const double P = (a1 * A[x] + a2 * B[x]) / zeta;
    const double PA = P - A[x], PB = P - B[x], X = A[x] - B[x];
    d2 += X * X;
    os1d<LA, LB>(PA, PB, inv2p, S[x]);
    if (KIN) {
      T[x][0][0] = xi * (1.0 - 2.0 * xi * X * X);
#pragma unroll
      for (int i = 0; i < LA; ++i) {
        double v = PA * T[x][i][0] + 2.0 * xi * S[x][i + 1][0];
        if (i > 0)
          v += i * inv2p * T[x][i - 1][0] -
               2.0 * xi * (i / (2.0 * a1)) * S[x][i - 1][0];
        T[x][i + 1][0] = v;
      }
#pragma unroll
      for (int j = 0; j < LB; ++j)
#pragma unroll
        for (int i = 0; i <= LA; ++i) {
          double v = PB * T[x][i][j] + 2.0 * xi * S[x][i][j + 1];
          if (i > 0) v += i * inv2p * T[x][i - 1][j];
          if (j > 0)
            v += j * inv2p * T[x][i][j - 1] -
                 2.0 * xi * (j / (2.0 * a2)) * S[x][i][j - 1];
          T[x][i][j + 1] = v;
        }
    }
  }
  const double pref = pow(kPi / zeta, 1.5) * exp(-xi * d2);
  double pc[ncart(LA) * ncart(LB)];
#pragma unroll
  for (int p = 0; p < ncart(LA); ++p)
#pragma unroll
    for (int q = 0; q < ncart(LB); ++q) {
      const int ax = cart_exp(p, 0), ay = cart_exp(p, 1), az = cart_exp(p, 2);
      const int bx = cart_exp(q, 0), by = cart_exp(q, 1), bz = cart_exp(q, 2);
      double v;
      if (KIN)
        v = T[0][ax][bx] * S[1][ay][by] * S[2][az][bz] +
            S[0][ax][bx] * T[1][ay][by] * S[2][az][bz] +
            S[0][ax][bx] * S[1][ay][by] * T[2][az][bz];
      else
        v = S[0][ax][bx] * S[1][ay][by] * S[2][az][bz];
      pc[p * ncart(LB) + q] = pref * v;
    }
  cart_to_sh<LA, LB>(pc, out);
}

// (alpha^2 / 8) with alpha the fine structure constant 7.2973525693e-3,
// the prefactor (fineStructure * 0.001)^2 / 8 of gaussIntegrals.f90:39118.
constexpr double kFineStructure = 7.2973525693 * 0.001;
constexpr double kMassVelPref = kFineStructure * kFineStructure / 8.0;

// One axis of the second derivative d^2/dx^2 x^i e^{-a x^2}
//   = i(i-1) x^{i-2} - 2a(2i+1) x^i + 4a^2 x^{i+2}
// taken on the left (atom 1), the right (atom 2) or both sides of the
// overlap table S (which runs two orders past the class on each side).
template <int IA, int JB>
__device__ __forceinline__ double d2_left(const double S[IA + 1][JB + 1],
                                          int i, int j, double a) {
  double v = -2.0 * a * (2 * i + 1) * S[i][j] + 4.0 * a * a * S[i + 2][j];
  if (i >= 2) v += i * (i - 1.0) * S[i - 2][j];
  return v;
}

template <int IA, int JB>
__device__ __forceinline__ double d2_right(const double S[IA + 1][JB + 1],
                                           int i, int j, double b) {
  double v = -2.0 * b * (2 * j + 1) * S[i][j] + 4.0 * b * b * S[i][j + 2];
  if (j >= 2) v += j * (j - 1.0) * S[i][j - 2];
  return v;
}

template <int IA, int JB>
__device__ __forceinline__ double d2_both(const double S[IA + 1][JB + 1],
                                          int i, int j, double a, double b) {
  double v = -2.0 * a * (2 * i + 1) * d2_right<IA, JB>(S, i, j, b) +
             4.0 * a * a * d2_right<IA, JB>(S, i + 2, j, b);
  if (i >= 2) v += i * (i - 1.0) * d2_right<IA, JB>(S, i - 2, j, b);
  return v;
}

// Mass-velocity block scale * <a|nabla^4|b> between primitives a1 at A and
// a2 at B (scale = kMassVelPref gives massvel2CIntg's sh; the build passes
// its negative, the sign the reference accumulates it with,
// integrals.F90:1440-1447).  nabla^4 is taken as <nabla^2 a|nabla^2 b>,
//   sum_x U_x S_y S_z + sum_{x != y} L_x R_y S_z,
// whose terms carry the size of the result; the reference's recursion seeds
// on 16 a2^4 <r_B^4> - 80 a2^3 <r_B^2> + 60 a2^2, which cancels to a value
// of order a1 a2 when a1 << a2.  s, p and d classes only (registers).
template <int LA, int LB>
__device__ void prim_mv(double a1, double a2, const double *A, const double *B,
                        double scale, double *out) {
  const double zeta = a1 + a2, xi = a1 * a2 / zeta, inv2p = 1.0 / (2.0 * zeta);
  // per axis: S, L (left d^2), R (right d^2), U (both) for i <= LA, j <= LB;
  // the extended overlap table lives only while its axis is formed
  double t[4][3][LA + 1][LB + 1];
  double d2 = 0.0;
#pragma unroll
  for (int x = 0; x < 3; ++x) {
    const double P = (a1 * A[x] + a2 * B[x]) / zeta;
    const double X = A[x] - B[x];
    d2 += X * X;
    double S[LA + 3][LB + 3];
    os1d<LA + 2, LB + 2>(P - A[x], P - B[x], inv2p, S);
#pragma unroll
    for (int i = 0; i <= LA; ++i)
#pragma unroll
      for (int j = 0; j <= LB; ++j) {
        t[0][x][i][j] = S[i][j];
        t[1][x][i][j] = d2_left<LA + 2, LB + 2>(S, i, j, a1);
        t[2][x][i][j] = d2_right<LA + 2, LB + 2>(S, i, j, a2);
        t[3][x][i][j] = d2_both<LA + 2, LB + 2>(S, i, j, a1, a2);
      }
  }
  const double pref = scale * pow(kPi / zeta, 1.5) * exp(-xi * d2);
  // one Cartesian pair, evaluated where a harmonic component needs it
  auto cart = [&](int p, int q) {
    const int i0 = cart_exp(p, 0), i1 = cart_exp(p, 1), i2 = cart_exp(p, 2);
    const int j0 = cart_exp(q, 0), j1 = cart_exp(q, 1), j2 = cart_exp(q, 2);
    const double s0 = t[0][0][i0][j0], s1 = t[0][1][i1][j1], s2 = t[0][2][i2][j2];
    const double l0 = t[1][0][i0][j0], l1 = t[1][1][i1][j1], l2 = t[1][2][i2][j2];
    const double r0 = t[2][0][i0][j0], r1 = t[2][1][i1][j1], r2 = t[2][2][i2][j2];
    const double u0 = t[3][0][i0][j0], u1 = t[3][1][i1][j1], u2 = t[3][2][i2][j2];
    double v = u0 * s1 * s2 + s0 * u1 * s2 + s0 * s1 * u2;
    v += (l0 * r1 + r0 * l1) * s2 + (l0 * r2 + r0 * l2) * s1 + (l1 * r2 + r1 * l2) * s0;
    return pref * v;
  };
#pragma unroll
  for (int s1 = 0; s1 < nsh(LA); ++s1)
#pragma unroll
    for (int s2 = 0; s2 < nsh(LB); ++s2) {
      double v = 0.0;
#pragma unroll
      for (int k1 = 0; k1 < 3; ++k1) {
        if (k1 >= sh_nterm(s1)) break;
#pragma unroll
        for (int k2 = 0; k2 < 3; ++k2) {
          if (k2 >= sh_nterm(s2)) break;
          v += sh_coef(s1, k1) * sh_coef(s2, k2) * cart(sh_cart(s1, k1), sh_cart(s2, k2));
        }
      }
      out[s1 * nsh(LB) + s2] = v;
    }
}

// Momentum <a|d/dx_c|b> (DIP = false) or dipole <a|(r - C)_c|b> (DIP =
// true) blocks for the three components c, written to out + c * cstride.
// The operator goes into the component's 1D factor of the overlap table:
//   dipole: (x - C_x) = x_B + (B_x - C_x) on atom 2's side;
//   momentum: d/dx x^j e^{-a x^2} = j x^{j-1} - 2 a x^{j+1} on atom 2's
//   side, or minus the same on atom 1's side (integration by parts), on the
//   side of the smaller exponent, so that the seed is formed from whichever
//   of PA = P - A and PB = P - B has not cancelled (the reference seeds
//   with 2 a1 PA S, gaussIntegrals.f90:23080-23082).
template <bool DIP, int IA, int JB>
__device__ __forceinline__ double vec_factor(const double S[IA + 1][JB + 1],
                                             int i, int j, bool left, double a1,
                                             double a2, double BC) {
  if (DIP) return S[i][j + 1] + BC * S[i][j];
  if (left) return 2.0 * a1 * S[i + 1][j] - (i > 0 ? i * S[i - 1][j] : 0.0);
  return -2.0 * a2 * S[i][j + 1] + (j > 0 ? j * S[i][j - 1] : 0.0);
}

// s, p and d classes: bounds known at compile time, tables in registers.
template <int LA, int LB, bool DIP>
__device__ void prim_vec(double a1, double a2, const double *A, const double *B,
                         const double *C, double *out, long long cstride) {
  const double zeta = a1 + a2, xi = a1 * a2 / zeta, inv2p = 1.0 / (2.0 * zeta);
  const bool left = a1 <= a2;
  double S[3][LA + 1][LB + 1], D[3][LA + 1][LB + 1];
  double d2 = 0.0;
#pragma unroll
  for (int x = 0; x < 3; ++x) {
    const double P = (a1 * A[x] + a2 * B[x]) / zeta;
    const double X = A[x] - B[x];
    d2 += X * X;
    double T[LA + 2][LB + 2];
    os1d<LA + 1, LB + 1>(P - A[x], P - B[x], inv2p, T);
    const double BC = DIP ? B[x] - C[x] : 0.0;
#pragma unroll
    for (int i = 0; i <= LA; ++i)
#pragma unroll
      for (int j = 0; j <= LB; ++j) {
        S[x][i][j] = T[i][j];
        D[x][i][j] = vec_factor<DIP, LA + 1, LB + 1>(T, i, j, left, a1, a2, BC);
      }
  }
  const double pref = pow(kPi / zeta, 1.5) * exp(-xi * d2);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    auto cart = [&](int p, int q) {
      double v = pref;
#pragma unroll
      for (int x = 0; x < 3; ++x) {
        const int i = cart_exp(p, x), j = cart_exp(q, x);
        v *= (x == c) ? D[x][i][j] : S[x][i][j];
      }
      return v;
    };
#pragma unroll
    for (int s1 = 0; s1 < nsh(LA); ++s1)
#pragma unroll
      for (int s2 = 0; s2 < nsh(LB); ++s2) {
        double v = 0.0;
#pragma unroll
        for (int k1 = 0; k1 < 3; ++k1) {
          if (k1 >= sh_nterm(s1)) break;
#pragma unroll
          for (int k2 = 0; k2 < 3; ++k2) {
            if (k2 >= sh_nterm(s2)) break;
            v += sh_coef(s1, k1) * sh_coef(s2, k2) * cart(sh_cart(s1, k1), sh_cart(s2, k2));
          }
        }
        out[c * cstride + s1 * nsh(LB) + s2] = v;
      }
  }
}

// ---------------------------------------------- McMurchie-Davidson 3C --
// Hermite expansion coefficients of one axis:
// E^{00}_0 = 1, E^{i+1,j}_t = E^{ij}_{t-1}/(2p) + PA E^{ij}_t + (t+1) E^{ij}_{t+1}
// and likewise for j with PB.
template <int LA, int LB>
__device__ __forceinline__ void hermite_e(double PA, double PB, double inv2p,
                                          double E[LA + 1][LB + 1][LA + LB + 1]) {
#pragma unroll
  for (int i = 0; i <= LA; ++i)
#pragma unroll
    for (int j = 0; j <= LB; ++j)
#pragma unroll
      for (int t = 0; t <= LA + LB; ++t) {
        double v;
        if (t > i + j) {
          v = 0.0;
        } else if (i == 0 && j == 0) {
          v = 1.0;
        } else if (i > 0) {
          v = PA * E[i - 1][j][t];
          if (t > 0) v += inv2p * E[i - 1][j][t - 1];
          if (t + 1 <= i - 1 + j) v += (t + 1) * E[i - 1][j][t + 1];
        } else {
          v = PB * E[i][j - 1][t];
          if (t > 0) v += inv2p * E[i][j - 1][t - 1];
          if (t + 1 <= i + j - 1) v += (t + 1) * E[i][j - 1][t + 1];
        }
        E[i][j][t] = v;
      }
}

// Accumulate one three-centre overlap term into Q: w * exp(-mu |X|^2)
// h_t(X) h_u(Y) h_v(Z), h_t = (d/dX)^t exp(-mu X^2) / exp(-mu X^2),
// h_{t+1} = -2 mu (X h_t + t h_{t-1}).
template <int L>
__device__ __forceinline__ void accumulate_overlap_q(const double X[3],
                                                     double mu, double w,
                                                     double Q[nherm(L)]) {
  double h[3][L + 1];
#pragma unroll
  for (int x = 0; x < 3; ++x) {
    h[x][0] = 1.0;
#pragma unroll
    for (int t = 0; t < L; ++t)
      h[x][t + 1] = -2.0 * mu * (X[x] * h[x][t] + (t > 0 ? t * h[x][t - 1] : 0.0));
  }
  const double g = w * exp(-mu * (X[0] * X[0] + X[1] * X[1] + X[2] * X[2]));
#pragma unroll
  for (int t = 0; t <= L; ++t)
#pragma unroll
    for (int u = 0; u <= L - t; ++u) {
      const double gtu = g * h[0][t] * h[1][u];
#pragma unroll
      for (int v = 0; v <= L - t - u; ++v)
        Q[herm_index(t, u, v)] += gtu * h[2][v];
    }
}

// Accumulate one nuclear term: w * d^{tuv}/dX^{tuv} of
// f(X) = exp(-mu |X|^2) F_0(nu |X|^2), the Gaussian-damped Coulomb
// potential integrated against the Hermite Gaussian of exponent p about P.
// With f = int_0^1 exp(-(mu + nu s^2)|X|^2) ds the Hermite recursion
//   R^n_{t+1,u,v} = t R^{n+1}_{t-1,u,v} + X R^{n+1}_{t,u,v}
// starts from R^n_000 = (-2)^n exp(-mu|X|^2) sum_k C(n,k) mu^{n-k} nu^k F_k.
template <int L>
__device__ __forceinline__ void accumulate_nuclear_q(const double X[3],
                                                     double mu, double nu,
                                                     double w,
                                                     double Q[nherm(L)]) {
  const double r2 = X[0] * X[0] + X[1] * X[1] + X[2] * X[2];
  double F[L + 1];
  boys_ref<L>(nu * r2, F);
  const double g = w * exp(-mu * r2);
  double R[L + 1][nherm(L)];
  // R^n_000
  {
    double mpow[L + 1], npow[L + 1];
    mpow[0] = 1.0;
    npow[0] = 1.0;
#pragma unroll
    for (int n = 1; n <= L; ++n) {
      mpow[n] = mpow[n - 1] * mu;
      npow[n] = npow[n - 1] * nu;
    }
    double sgn = 1.0;
#pragma unroll
    for (int n = 0; n <= L; ++n) {
      double s = 0.0, binom = 1.0;
#pragma unroll
      for (int k = 0; k <= n; ++k) {
        s += binom * mpow[n - k] * npow[k] * F[k];
        binom = binom * (n - k) / (k + 1);
      }
      R[n][0] = sgn * g * s;
      sgn *= -2.0;
    }
  }
#pragma unroll
  for (int tot = 1; tot <= L; ++tot)
#pragma unroll
    for (int t = tot; t >= 0; --t)
#pragma unroll
      for (int u = tot - t; u >= 0; --u) {
        const int v = tot - t - u;
        const int id = herm_index(t, u, v);
#pragma unroll
        for (int n = 0; n <= L - tot; ++n) {
          double val;
          if (t > 0) {
            val = X[0] * R[n + 1][herm_index(t - 1, u, v)];
            if (t > 1) val += (t - 1) * R[n + 1][herm_index(t - 2, u, v)];
          } else if (u > 0) {
            val = X[1] * R[n + 1][herm_index(t, u - 1, v)];
            if (u > 1) val += (u - 1) * R[n + 1][herm_index(t, u - 2, v)];
          } else {
            val = X[2] * R[n + 1][herm_index(t, u, v - 1)];
            if (v > 1) val += (v - 1) * R[n + 1][herm_index(t, u, v - 2)];
          }
          R[n][id] = val;
        }
      }
#pragma unroll
  for (int i = 0; i < nherm(L); ++i) Q[i] += R[0][i];
}

// Turn accumulated Hermite integrals Q into the sh block:
// pc(a, b) = pref * sum_tuv Ex[ax][bx][t] Ey[ay][by][u] Ez[az][bz][v] Q_tuv.
template <int LA, int LB>
__device__ void hermite_to_sh(const double *A, const double *B, double a1,
                              double a2, double pref,
                              const double Q[nherm(LA + LB)], double *out) {
  constexpr int L = LA + LB;
  const double zeta = a1 + a2, inv2p = 1.0 / (2.0 * zeta);
  double E[3][LA + 1][LB + 1][L + 1];
#pragma unroll
  for (int x = 0; x < 3; ++x) {
    const double P = (a1 * A[x] + a2 * B[x]) / zeta;
    hermite_e<LA, LB>(P - A[x], P - B[x], inv2p, E[x]);
  }
  double pc[ncart(LA) * ncart(LB)];
#pragma unroll
  for (int p = 0; p < ncart(LA); ++p)
#pragma unroll
    for (int q = 0; q < ncart(LB); ++q) {
      const int ax = cart_exp(p, 0), ay = cart_exp(p, 1), az = cart_exp(p, 2);
      const int bx = cart_exp(q, 0), by = cart_exp(q, 1), bz = cart_exp(q, 2);
      double s = 0.0;
#pragma unroll
      for (int t = 0; t <= L; ++t) {
        if (t > ax + bx) break;
#pragma unroll
        for (int u = 0; u <= L; ++u) {
          if (u > ay + by) break;
          const double etu = E[0][ax][bx][t] * E[1][ay][by][u];
#pragma unroll
          for (int v = 0; v <= L; ++v) {
            if (v > az + bz) break;
            s += etu * E[2][az][bz][v] * Q[herm_index(t, u, v)];
          }
        }
      }
      pc[p * ncart(LB) + q] = pref * s;
    }
  cart_to_sh<LA, LB>(pc, out);
}

// ------------------------------------------------ f classes, runtime loops --
// Classes with an f side are rare (no f functions in the measured
// workloads) and their fully unrolled forms are very large, so they share
// one implementation with runtime class arguments and small local arrays.
constexpr int kMaxL = 6;
constexpr int kMaxHerm = nherm(kMaxL);  // 84

static __device__ __forceinline__ void cart_to_sh_rt(int la, int lb, const double *pc,
                                              double *out) {
  const int ncb = ncart(lb), nsa = nsh(la), nsb = nsh(lb);
#pragma unroll 1
  for (int s1 = 0; s1 < nsa; ++s1)
#pragma unroll 1
    for (int s2 = 0; s2 < nsb; ++s2) {
      double v = 0.0;
      for (int k1 = 0; k1 < sh_nterm(s1); ++k1)
        for (int k2 = 0; k2 < sh_nterm(s2); ++k2)
          v += sh_coef(s1, k1) * sh_coef(s2, k2) *
               pc[sh_cart(s1, k1) * ncb + sh_cart(s2, k2)];
      out[s1 * nsb + s2] = v;
    }
}

static __device__ __noinline__ void prim2c_rt(int la, int lb, bool kin, double a1,
                                       double a2, const double *A,
                                       const double *B, double *out) {
  const double zeta = a1 + a2, xi = a1 * a2 / zeta, inv2p = 1.0 / (2.0 * zeta);
  double S[3][4][4], T[3][4][4];
  double d2 = 0.0;
#pragma unroll 1
  for (int x = 0; x < 3; ++x) {
    const double P = (a1 * A[x] + a2 * B[x]) / zeta;
    const double PA = P - A[x], PB = P - B[x], X = A[x] - B[x];
    d2 += X * X;
    S[x][0][0] = 1.0;
    for (int i = 0; i < la; ++i)
      S[x][i + 1][0] = PA * S[x][i][0] + (i > 0 ? i * inv2p * S[x][i - 1][0] : 0.0);
    for (int j = 0; j < lb; ++j)
      for (int i = 0; i <= la; ++i) {
        double v = PB * S[x][i][j];
        if (i > 0) v += i * inv2p * S[x][i - 1][j];
        if (j > 0) v += j * inv2p * S[x][i][j - 1];
        S[x][i][j + 1] = v;
      }
    if (kin) {
      T[x][0][0] = xi * (1.0 - 2.0 * xi * X * X);
      for (int i = 0; i < la; ++i) {
        double v = PA * T[x][i][0] + 2.0 * xi * S[x][i + 1][0];
        if (i > 0)
          v += i * inv2p * T[x][i - 1][0] -
               2.0 * xi * (i / (2.0 * a1)) * S[x][i - 1][0];
        T[x][i + 1][0] = v;
      }
      for (int j = 0; j < lb; ++j)
        for (int i = 0; i <= la; ++i) {
          double v = PB * T[x][i][j] + 2.0 * xi * S[x][i][j + 1];
          if (i > 0) v += i * inv2p * T[x][i - 1][j];
          if (j > 0)
            v += j * inv2p * T[x][i][j - 1] -
                 2.0 * xi * (j / (2.0 * a2)) * S[x][i][j - 1];
          T[x][i][j + 1] = v;
        }
    }
  }
  const double pref = pow(kPi / zeta, 1.5) * exp(-xi * d2);
  double pc[400];
  const int nca = ncart(la), ncb = ncart(lb);
  for (int p = 0; p < nca; ++p)
    for (int q = 0; q < ncb; ++q) {
      const int ax = cart_exp(p, 0), ay = cart_exp(p, 1), az = cart_exp(p, 2);
      const int bx = cart_exp(q, 0), by = cart_exp(q, 1), bz = cart_exp(q, 2);
      double v;
      if (kin)
        v = T[0][ax][bx] * S[1][ay][by] * S[2][az][bz] +
            S[0][ax][bx] * T[1][ay][by] * S[2][az][bz] +
            S[0][ax][bx] * S[1][ay][by] * T[2][az][bz];
      else
        v = S[0][ax][bx] * S[1][ay][by] * S[2][az][bz];
      pc[p * ncb + q] = pref * v;
    }
  cart_to_sh_rt(la, lb, pc, out);
}

// prim_mv for the f classes, with runtime loops over tables in local
// memory (a fully unrolled f-d or f-f block does not fit the registers).
static __device__ __noinline__ void prim_mv_rt(int la, int lb, double a1,
                                               double a2, const double *A,
                                               const double *B, double scale,
                                               double *out) {
  const double zeta = a1 + a2, xi = a1 * a2 / zeta, inv2p = 1.0 / (2.0 * zeta);
  double t[4][3][4][4];
  double d2 = 0.0;
#pragma unroll 1
  for (int x = 0; x < 3; ++x) {
    const double P = (a1 * A[x] + a2 * B[x]) / zeta;
    const double X = A[x] - B[x];
    d2 += X * X;
    double S[6][6];
    os1d<5, 5>(P - A[x], P - B[x], inv2p, S);
#pragma unroll 1
    for (int i = 0; i <= la; ++i)
#pragma unroll 1
      for (int j = 0; j <= lb; ++j) {
        t[0][x][i][j] = S[i][j];
        t[1][x][i][j] = d2_left<5, 5>(S, i, j, a1);
        t[2][x][i][j] = d2_right<5, 5>(S, i, j, a2);
        t[3][x][i][j] = d2_both<5, 5>(S, i, j, a1, a2);
      }
  }
  const double pref = scale * pow(kPi / zeta, 1.5) * exp(-xi * d2);
  double pc[ncart(3) * ncart(3)];
  const int nca = ncart(la), ncb = ncart(lb);
#pragma unroll 1
  for (int p = 0; p < nca; ++p)
#pragma unroll 1
    for (int q = 0; q < ncb; ++q) {
      double s[3], l[3], r[3], u[3];
      for (int x = 0; x < 3; ++x) {
        const int i = cart_exp(p, x), j = cart_exp(q, x);
        s[x] = t[0][x][i][j];
        l[x] = t[1][x][i][j];
        r[x] = t[2][x][i][j];
        u[x] = t[3][x][i][j];
      }
      double v = u[0] * s[1] * s[2] + s[0] * u[1] * s[2] + s[0] * s[1] * u[2];
      v += (l[0] * r[1] + r[0] * l[1]) * s[2] + (l[0] * r[2] + r[0] * l[2]) * s[1] +
           (l[1] * r[2] + r[1] * l[2]) * s[0];
      pc[p * ncb + q] = pref * v;
    }
  cart_to_sh_rt(la, lb, pc, out);
}

// prim_vec for the f classes: runtime loops, tables in local memory.
template <bool DIP>
__device__ __noinline__ void prim_vec_rt(int la, int lb, double a1, double a2,
                                         const double *A, const double *B,
                                         const double *C, double *out,
                                         long long cstride) {
  const double zeta = a1 + a2, xi = a1 * a2 / zeta, inv2p = 1.0 / (2.0 * zeta);
  const bool left = a1 <= a2;
  double S[3][4][4], D[3][4][4];
  double d2 = 0.0;
#pragma unroll 1
  for (int x = 0; x < 3; ++x) {
    const double P = (a1 * A[x] + a2 * B[x]) / zeta;
    const double X = A[x] - B[x];
    d2 += X * X;
    double T[5][5];
    os1d<4, 4>(P - A[x], P - B[x], inv2p, T);
    const double BC = DIP ? B[x] - C[x] : 0.0;
#pragma unroll 1
    for (int i = 0; i <= la; ++i)
#pragma unroll 1
      for (int j = 0; j <= lb; ++j) {
        S[x][i][j] = T[i][j];
        D[x][i][j] = vec_factor<DIP, 4, 4>(T, i, j, left, a1, a2, BC);
      }
  }
  const double pref = pow(kPi / zeta, 1.5) * exp(-xi * d2);
  const int nca = ncart(la), ncb = ncart(lb), nsa = nsh(la), nsb = nsh(lb);
  double pc[ncart(3) * ncart(3)];
#pragma unroll 1
  for (int c = 0; c < 3; ++c) {
#pragma unroll 1
    for (int p = 0; p < nca; ++p)
#pragma unroll 1
      for (int q = 0; q < ncb; ++q) {
        double v = pref;
        for (int x = 0; x < 3; ++x) {
          const int i = cart_exp(p, x), j = cart_exp(q, x);
          v *= (x == c) ? D[x][i][j] : S[x][i][j];
        }
        pc[p * ncb + q] = v;
      }
    double blk[256];
    cart_to_sh_rt(la, lb, pc, blk);
#pragma unroll 1
    for (int e = 0; e < nsa * nsb; ++e) out[c * cstride + e] = blk[e];
  }
}

// The plane-wave overlap for one wave vector q with compile-time classes
// (s, p, d): the same complex-shifted recursion as prim_kov below, its
// tables and the Cartesian products unrolled into registers.
template <int LA, int LB>
__device__ void prim_kov_t(double a1, double a2, const double *A, const double *B,
                           const double *q, double *out_re, double *out_im) {
  const double zeta = a1 + a2, xi = a1 * a2 / zeta, inv2p = 1.0 / (2.0 * zeta);
  double Sr[3][LA + 1][LB + 1], Si[3][LA + 1][LB + 1], fr[3], fi[3];
#pragma unroll
  for (int x = 0; x < 3; ++x) {
    const double P = (a1 * A[x] + a2 * B[x]) / zeta, X = A[x] - B[x];
    const double ar = P - A[x], br = P - B[x], sh = -q[x] * inv2p;
    Sr[x][0][0] = 1.0;
    Si[x][0][0] = 0.0;
#pragma unroll
    for (int i = 0; i < LA; ++i) {
      double vr = ar * Sr[x][i][0] - sh * Si[x][i][0];
      double vi = ar * Si[x][i][0] + sh * Sr[x][i][0];
      if (i > 0) {
        vr += i * inv2p * Sr[x][i - 1][0];
        vi += i * inv2p * Si[x][i - 1][0];
      }
      Sr[x][i + 1][0] = vr;
      Si[x][i + 1][0] = vi;
    }
#pragma unroll
    for (int j = 0; j < LB; ++j)
#pragma unroll
      for (int i = 0; i <= LA; ++i) {
        double vr = br * Sr[x][i][j] - sh * Si[x][i][j];
        double vi = br * Si[x][i][j] + sh * Sr[x][i][j];
        if (i > 0) {
          vr += i * inv2p * Sr[x][i - 1][j];
          vi += i * inv2p * Si[x][i - 1][j];
        }
        if (j > 0) {
          vr += j * inv2p * Sr[x][i][j - 1];
          vi += j * inv2p * Si[x][i][j - 1];
        }
        Sr[x][i][j + 1] = vr;
        Si[x][i][j + 1] = vi;
      }
    const double mag = sqrt(kPi / zeta) * exp(-xi * X * X) * exp(-q[x] * q[x] / (4.0 * zeta));
    double sn, cs;
    sincos(q[x] * P, &sn, &cs);
    fr[x] = mag * cs;
    fi[x] = -mag * sn;
  }
  double pcr[ncart(LA) * ncart(LB)], pci[ncart(LA) * ncart(LB)];
#pragma unroll
  for (int p = 0; p < ncart(LA); ++p)
#pragma unroll
    for (int c = 0; c < ncart(LB); ++c) {
      double vr = 1.0, vi = 0.0;
#pragma unroll
      for (int x = 0; x < 3; ++x) {
        const int i = cart_exp(p, x), j = cart_exp(c, x);
        const double gr = Sr[x][i][j] * fr[x] - Si[x][i][j] * fi[x];
        const double gi = Sr[x][i][j] * fi[x] + Si[x][i][j] * fr[x];
        const double nr = vr * gr - vi * gi, ni = vr * gi + vi * gr;
        vr = nr;
        vi = ni;
      }
      pcr[p * ncart(LB) + c] = vr;
      pci[p * ncart(LB) + c] = vi;
    }
  cart_to_sh<LA, LB>(pcr, out_re);
  cart_to_sh<LA, LB>(pci, out_im);
}


// Overlap with a plane wave, <a|exp(-i q.r)|b> (KOverlap2CIntg), complex,
// as two real blocks.  The product Gaussian times exp(-i q x) is
// exp(-i q P - q^2/(4p)) times a Gaussian about P' = P - i q/(2p): the 1D
// recursion runs with the complex PA' = PA - i q/(2p), PB' = PB - i q/(2p)
// and each axis carries sqrt(pi/p) exp(-xi X^2) exp(-q^2/(4p)) exp(-i q P).
// Runtime loops (every class; the build runs once per optical run).
static __device__ __noinline__ void prim_kov(int la, int lb, double a1, double a2,
                                             const double *A, const double *B,
                                             const double *q, double *out_re,
                                             double *out_im) {
  const double zeta = a1 + a2, xi = a1 * a2 / zeta, inv2p = 1.0 / (2.0 * zeta);
  double Sr[3][4][4], Si[3][4][4], fr[3], fi[3];
#pragma unroll 1
  for (int x = 0; x < 3; ++x) {
    const double P = (a1 * A[x] + a2 * B[x]) / zeta, X = A[x] - B[x];
    const double ar = P - A[x], br = P - B[x], sh = -q[x] * inv2p;
    Sr[x][0][0] = 1.0;
    Si[x][0][0] = 0.0;
    for (int i = 0; i < la; ++i) {
      double vr = ar * Sr[x][i][0] - sh * Si[x][i][0];
      double vi = ar * Si[x][i][0] + sh * Sr[x][i][0];
      if (i > 0) {
        vr += i * inv2p * Sr[x][i - 1][0];
        vi += i * inv2p * Si[x][i - 1][0];
      }
      Sr[x][i + 1][0] = vr;
      Si[x][i + 1][0] = vi;
    }
    for (int j = 0; j < lb; ++j)
      for (int i = 0; i <= la; ++i) {
        double vr = br * Sr[x][i][j] - sh * Si[x][i][j];
        double vi = br * Si[x][i][j] + sh * Sr[x][i][j];
        if (i > 0) {
          vr += i * inv2p * Sr[x][i - 1][j];
          vi += i * inv2p * Si[x][i - 1][j];
        }
        if (j > 0) {
          vr += j * inv2p * Sr[x][i][j - 1];
          vi += j * inv2p * Si[x][i][j - 1];
        }
        Sr[x][i][j + 1] = vr;
        Si[x][i][j + 1] = vi;
      }
    const double mag = sqrt(kPi / zeta) * exp(-xi * X * X) * exp(-q[x] * q[x] / (4.0 * zeta));
    double sn, cs;
    sincos(q[x] * P, &sn, &cs);
    fr[x] = mag * cs;
    fi[x] = -mag * sn;
  }
  double pcr[ncart(3) * ncart(3)], pci[ncart(3) * ncart(3)];
  const int nca = ncart(la), ncb = ncart(lb);
#pragma unroll 1
  for (int p = 0; p < nca; ++p)
#pragma unroll 1
    for (int c = 0; c < ncb; ++c) {
      double vr = 1.0, vi = 0.0;
      for (int x = 0; x < 3; ++x) {
        const int i = cart_exp(p, x), j = cart_exp(c, x);
        const double gr = Sr[x][i][j] * fr[x] - Si[x][i][j] * fi[x];
        const double gi = Sr[x][i][j] * fi[x] + Si[x][i][j] * fr[x];
        const double nr = vr * gr - vi * gi, ni = vr * gi + vi * gr;
        vr = nr;
        vi = ni;
      }
      pcr[p * ncb + c] = vr;
      pci[p * ncb + c] = vi;
    }
  cart_to_sh_rt(la, lb, pcr, out_re);
  cart_to_sh_rt(la, lb, pci, out_im);
}

static __device__ __noinline__ void accumulate_overlap_q_rt(int L, const double *X,
                                                     double mu, double w,
                                                     double *Q) {
  double h[3][kMaxL + 1];
  for (int x = 0; x < 3; ++x) {
    h[x][0] = 1.0;
    for (int t = 0; t < L; ++t)
      h[x][t + 1] = -2.0 * mu * (X[x] * h[x][t] + (t > 0 ? t * h[x][t - 1] : 0.0));
  }
  const double g = w * exp(-mu * (X[0] * X[0] + X[1] * X[1] + X[2] * X[2]));
  for (int t = 0; t <= L; ++t)
    for (int u = 0; u <= L - t; ++u) {
      const double gtu = g * h[0][t] * h[1][u];
      for (int v = 0; v <= L - t - u; ++v) Q[herm_index(t, u, v)] += gtu * h[2][v];
    }
}

static __device__ __noinline__ void accumulate_nuclear_q_rt(int L, const double *X,
                                                     double mu, double nu,
                                                     double w, double *Q) {
  const double r2 = X[0] * X[0] + X[1] * X[1] + X[2] * X[2];
  double F[kMaxL + 1];
  boys_ref<kMaxL>(nu * r2, F);
  const double g = w * exp(-mu * r2);
  double R[kMaxL + 1][kMaxHerm];
  double mpow[kMaxL + 1], npow[kMaxL + 1];
  mpow[0] = npow[0] = 1.0;
  for (int n = 1; n <= L; ++n) {
    mpow[n] = mpow[n - 1] * mu;
    npow[n] = npow[n - 1] * nu;
  }
  double sgn = 1.0;
  for (int n = 0; n <= L; ++n) {
    double s = 0.0, binom = 1.0;
    for (int k = 0; k <= n; ++k) {
      s += binom * mpow[n - k] * npow[k] * F[k];
      binom = binom * (n - k) / (k + 1);
    }
    R[n][0] = sgn * g * s;
    sgn *= -2.0;
  }
  for (int tot = 1; tot <= L; ++tot)
    for (int t = tot; t >= 0; --t)
      for (int u = tot - t; u >= 0; --u) {
        const int v = tot - t - u, id = herm_index(t, u, v);
        for (int n = 0; n <= L - tot; ++n) {
          double val;
          if (t > 0) {
            val = X[0] * R[n + 1][herm_index(t - 1, u, v)];
            if (t > 1) val += (t - 1) * R[n + 1][herm_index(t - 2, u, v)];
          } else if (u > 0) {
            val = X[1] * R[n + 1][herm_index(t, u - 1, v)];
            if (u > 1) val += (u - 1) * R[n + 1][herm_index(t, u - 2, v)];
          } else {
            val = X[2] * R[n + 1][herm_index(t, u, v - 1)];
            if (v > 1) val += (v - 1) * R[n + 1][herm_index(t, u, v - 2)];
          }
          R[n][id] = val;
        }
      }
  for (int i = 0; i < nherm(L); ++i) Q[i] += R[0][i];
}

static __device__ __noinline__ void hermite_to_sh_rt(int la, int lb, const double *A,
                                              const double *B, double a1,
                                              double a2, double pref,
                                              const double *Q, double *out) {
  const int L = la + lb;
  const double zeta = a1 + a2, inv2p = 1.0 / (2.0 * zeta);
  double E[3][4][4][kMaxL + 1];
  for (int x = 0; x < 3; ++x) {
    const double P = (a1 * A[x] + a2 * B[x]) / zeta;
    const double PA = P - A[x], PB = P - B[x];
    for (int i = 0; i <= la; ++i)
      for (int j = 0; j <= lb; ++j)
        for (int t = 0; t <= L; ++t) {
          double v;
          if (t > i + j) v = 0.0;
          else if (i == 0 && j == 0) v = 1.0;
          else if (i > 0) {
            v = PA * E[x][i - 1][j][t];
            if (t > 0) v += inv2p * E[x][i - 1][j][t - 1];
            if (t + 1 <= i - 1 + j) v += (t + 1) * E[x][i - 1][j][t + 1];
          } else {
            v = PB * E[x][i][j - 1][t];
            if (t > 0) v += inv2p * E[x][i][j - 1][t - 1];
            if (t + 1 <= i + j - 1) v += (t + 1) * E[x][i][j - 1][t + 1];
          }
          E[x][i][j][t] = v;
        }
  }
  double pc[400];
  const int nca = ncart(la), ncb = ncart(lb);
  for (int p = 0; p < nca; ++p)
    for (int q = 0; q < ncb; ++q) {
      const int ax = cart_exp(p, 0), ay = cart_exp(p, 1), az = cart_exp(p, 2);
      const int bx = cart_exp(q, 0), by = cart_exp(q, 1), bz = cart_exp(q, 2);
      double s = 0.0;
      for (int t = 0; t <= ax + bx; ++t)
        for (int u = 0; u <= ay + by; ++u) {
          const double etu = E[0][ax][bx][t] * E[1][ay][by][u];
          for (int v = 0; v <= az + bz; ++v)
            s += etu * E[2][az][bz][v] * Q[herm_index(t, u, v)];
        }
      pc[p * ncb + q] = pref * s;
    }
  cart_to_sh_rt(la, lb, pc, out);
}

}  // namespace imago
