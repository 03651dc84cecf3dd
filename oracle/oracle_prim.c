/*
 * oracle_prim.c -- CPU restatement of the reference's primitive integrals.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * The reference evaluates each primitive pair with straight-line
 * Obara-Saika code emitted by src/scripts/osrecurintg.py into
 * src/imago/gaussIntegrals.f90.  This file computes the same quantities from
 * the recursions themselves, written independently:
 *
 *   overlap2CIntg  (gaussIntegrals.f90:26-4420)    <a|b>
 *   kinetic2CIntg  (gaussIntegrals.f90:4422-11622) <a|-1/2 nabla^2|b>
 *   massvel2CIntg  (gaussIntegrals.f90:39070-49402) (alpha^2/8)<a|nabla^4|b>
 *   momentum2CIntg (gaussIntegrals.f90:23041-39068) <a|d/dx_c|b>, c = x,y,z
 *   dipole3CIntg   (gaussIntegrals.f90:49404-65510) <a|(r - C)_c|b>
 *   KOverlap2CIntg (gaussIntegrals.f90:129408-135102) <a|exp(-i dK.r)|b>
 *   electron3CIntg (gaussIntegrals.f90:11624-16023) <a|exp(-a3 r_C^2)|b>
 *   nuclear3CIntg  (gaussIntegrals.f90:16223-23039) <a|exp(-a3 r_C^2)/r_C|b>
 *
 * over unnormalised Cartesian Gaussians, then combined into the reference's
 * real-solid-harmonic order (sh(16,16): 1 s; 2 x; 3 y; 4 z; 5 xy; 6 xz;
 * 7 yz; 8 xx-yy; 9 2zz-xx-yy; 10 xyz; 11 xxz-yyz; 12 xxx-3yyx;
 * 13 3xxy-yyy; 14 2zzz-3xxz-3yyz; 15 4zzx-xxx-yyx; 16 4zzy-xxy-yyy, the
 * table at src/scripts/osrecurintg.py:332-426).  A class l on one side
 * means all functions up to l (nsh = 1, 4, 9, 16), as the reference's
 * lmAlphaIndex classes do (basis.f90:138-146).
 *
 * The Boys function restates gaussIntegrals.f90:16080-16221 branch for
 * branch, including its single-precision series constants.
 */
#include <math.h>
#include <string.h>

#include "oracle.h"

static const double ORC_PI = 3.141592653589793; /* constants.f90:36 */

/* Cartesian components in the reference's pc order (pc(20,20): 1 s; 2 x;
 * 3 y; 4 z; 5 xx; 6 yy; 7 zz; 8 xy; 9 xz; 10 yz; 11 xyz; 12 xxy; 13 xxz;
 * 14 yyx; 15 yyz; 16 zzx; 17 zzy; 18 xxx; 19 yyy; 20 zzz). */
static const int CART[20][3] = {
    {0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0}, {0, 2, 0},
    {0, 0, 2}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}, {2, 1, 0},
    {2, 0, 1}, {1, 2, 0}, {0, 2, 1}, {1, 0, 2}, {0, 1, 2}, {3, 0, 0},
    {0, 3, 0}, {0, 0, 3}};
static const int NCART[4] = {1, 4, 10, 20};
static const int NSH[4] = {1, 4, 9, 16};

/* sh component -> linear combination of pc components (0-based). */
typedef struct {
  int n;
  double c[3];
  int p[3];
} shmap;
static const shmap SHC[16] = {
    {1, {1, 0, 0}, {0, 0, 0}},    {1, {1, 0, 0}, {1, 0, 0}},
    {1, {1, 0, 0}, {2, 0, 0}},    {1, {1, 0, 0}, {3, 0, 0}},
    {1, {1, 0, 0}, {7, 0, 0}},    {1, {1, 0, 0}, {8, 0, 0}},
    {1, {1, 0, 0}, {9, 0, 0}},    {2, {1, -1, 0}, {4, 5, 0}},
    {3, {2, -1, -1}, {6, 4, 5}},  {1, {1, 0, 0}, {10, 0, 0}},
    {2, {1, -1, 0}, {12, 14, 0}}, {2, {1, -3, 0}, {17, 13, 0}},
    {2, {3, -1, 0}, {11, 18, 0}}, {3, {2, -3, -3}, {19, 12, 14}},
    {3, {4, -1, -1}, {15, 17, 13}}, {3, {4, -1, -1}, {16, 11, 18}}};

static void cart_to_sh(const double pc[20][20], int la, int lb, double *sh) {
  memset(sh, 0, sizeof(double) * 256);
  for (int i = 0; i < NSH[la]; ++i)
    for (int j = 0; j < NSH[lb]; ++j) {
      double s = 0.0;
      for (int p = 0; p < SHC[i].n; ++p)
        for (int q = 0; q < SHC[j].n; ++q)
          s += SHC[i].c[p] * SHC[j].c[q] * pc[SHC[i].p[p]][SHC[j].p[q]];
      sh[i * 16 + j] = s;
    }
}

/* Boys function F_0..F_6 (gaussIntegrals.f90:16080-16221).  For
 * T <= 10E-2 (a default-REAL literal, so the threshold is the single
 * precision 0.1f) the reference sums seven terms of the series
 *   F_N(T) = 1/2 e^{-T} Gamma(N+1/2) sum_k T^k / Gamma(N+k+3/2)
 * with Gamma(n+1/2) written as default-REAL literals, i.e. rounded to
 * single precision; above it, the closed forms in erf(sqrt T) and exp(-T).
 * Both are kept here exactly, because the single-precision constants and
 * the closed-form cancellation move the values by up to ~1e-7 relative
 * from the exact function, and matrix elements must match the reference. */
static const float GAMMA_HALF_F[14] = {
    1.7724538509055161f, 0.88622692545275805f, 1.3293403881791370f,
    3.3233509704478426f, 11.631728396567450f,  52.342777784553533f,
    287.88527781504416f, 1871.2543057977896f,  14034.407293483402f,
    119292.46199460901f, 1133278.3889487833f,  11899423.083962219f,
    136843365.46556622f, 1710542068.3195722f};

void orc_boys(double T, double F[7]) {
  const double exp_T = exp(-T);
  const double sqrt_pi = sqrt(ORC_PI);
  const double erf_T = erf(sqrt(T));
  if (T <= (double)0.1f) {
    for (int N = 0; N <= 6; ++N) {
      double a[8];
      for (int k = 0; k < 8; ++k) a[k] = (double)GAMMA_HALF_F[N + k];
      /* integer powers as gfortran's power tree forms them */
      double T2 = T * T, T3 = T2 * T, T4 = T2 * T2;
      double T5 = T3 * T2, T6 = T3 * T3;
      F[N] = 0.5 * exp_T * a[0] *
             ((1 / a[1]) + (T / a[2]) + (T2 / a[3]) + (T3 / a[4]) +
              (T4 / a[5]) + (T5 / a[6]) + (T6 / a[7]));
    }
    return;
  }
  /* Closed forms.  For order m >= 1:
   *   F_m = c_m [ sqrt(pi) erf / (4^m T^{m+1/2})
   *               - e^{-T} sum_{k=1..m} (m-k+1)! / (4^{k-1} (2(m-k+1))! T^k) ]
   * with c_1 = 1, c_m = c_{m-1} (4m - 2); evaluated in the reference's
   * operation order. */
  F[0] = 0.5 * ((sqrt_pi / pow(T, 0.5)) * erf_T);
  static const double fact[14] = {1,       1,        2,         6,
                                  24,      120,      720,       5040,
                                  40320,   362880,   3628800,   39916800,
                                  479001600, 6227020800.0};
  double c = 1.0;
  for (int m = 1; m <= 6; ++m) {
    if (m > 1) c *= (double)(4 * m - 2);
    double p4m = 1.0;
    for (int q = 0; q < m; ++q) p4m *= 4.0;
    double erfterm = (sqrt_pi / (p4m * pow(T, (double)m + 0.5))) * erf_T;
    double s = 0.0;
    double p4k = 1.0;
    for (int k = 1; k <= m; ++k) {
      int r = m - k + 1;
      double num = fact[r];
      double den;
      double T2 = T * T, T3 = T2 * T;
      double Tk = k == 2 ? T2 : k == 3 ? T3 : k == 4 ? T2 * T2
                : k == 5 ? T3 * T2 : T3 * T3;
      if (k == 1)
        den = fact[2 * r] * T;
      else
        den = (p4k * fact[2 * r]) * Tk;
      double term = num / den;
      s = (k == 1) ? term : s + term;
      p4k *= 4.0;
    }
    double v = erfterm - exp_T * s;
    F[m] = (m == 1) ? v : c * v;
  }
}

/* 1D Obara-Saika overlap table S[i][j] (without the prefactor) for a
 * Gaussian product centred at P with exponent p: S[0][0] = 1,
 * S[i+1][j] = PA S[i][j] + (i S[i-1][j] + j S[i][j-1]) / (2p),
 * S[i][j+1] = PB S[i][j] + (i S[i-1][j] + j S[i][j-1]) / (2p). */
static void os_1d(double PA, double PB, double inv2p, int imax, int jmax,
                  double S[8][8]) {
  S[0][0] = 1.0;
  for (int i = 0; i < imax; ++i)
    S[i + 1][0] = PA * S[i][0] + (i > 0 ? i * inv2p * S[i - 1][0] : 0.0);
  for (int j = 0; j < jmax; ++j)
    for (int i = 0; i <= imax; ++i) {
      double v = PB * S[i][j];
      if (i > 0) v += i * inv2p * S[i - 1][j];
      if (j > 0) v += j * inv2p * S[i][j - 1];
      S[i][j + 1] = v;
    }
}

void orc_overlap2c(double a1, double a2, const double *A, const double *B,
                   int la, int lb, double *sh) {
  double zeta = a1 + a2, xi = a1 * a2 / zeta, d2 = 0.0;
  double S[3][8][8];
  for (int x = 0; x < 3; ++x) {
    double P = (a1 * A[x] + a2 * B[x]) / zeta;
    d2 += (A[x] - B[x]) * (A[x] - B[x]);
    os_1d(P - A[x], P - B[x], 1.0 / (2.0 * zeta), la, lb, S[x]);
  }
  double pref = pow(ORC_PI / zeta, 1.5) * exp(-xi * d2);
  double pc[20][20];
  for (int p = 0; p < NCART[la]; ++p)
    for (int q = 0; q < NCART[lb]; ++q)
      pc[p][q] = pref * S[0][CART[p][0]][CART[q][0]] *
                 S[1][CART[p][1]][CART[q][1]] * S[2][CART[p][2]][CART[q][2]];
  cart_to_sh(pc, la, lb, sh);
}

/* Kinetic energy by the Obara-Saika kinetic recursion in its separable
 * 1D form (each Cartesian factor of -1/2 nabla^2 acts on one axis):
 *   T_00 = xi (1 - 2 xi X^2),  X = A_x - B_x,
 *   T_{i+1,j} = PA T_ij + (i T_{i-1,j} + j T_{i,j-1})/(2p)
 *               + 2 xi (S_{i+1,j} - i/(2 a1) S_{i-1,j}),
 *   T_{i,j+1} = PB T_ij + (i T_{i-1,j} + j T_{i,j-1})/(2p)
 *               + 2 xi (S_{i,j+1} - j/(2 a2) S_{i,j-1}),
 * then KE = pref (Tx Sy Sz + Sx Ty Sz + Sx Sy Tz), which for s-s is the
 * reference's preFactorKE = xi (3 - 2 xi d^2) S (gaussIntegrals.f90:4461). */
void orc_kinetic2c(double a1, double a2, const double *A, const double *B,
                   int la, int lb, double *sh) {
  double zeta = a1 + a2, xi = a1 * a2 / zeta, d2 = 0.0;
  double inv2p = 1.0 / (2.0 * zeta);
  double S[3][8][8], T[3][8][8];
  for (int x = 0; x < 3; ++x) {
    double P = (a1 * A[x] + a2 * B[x]) / zeta;
    double PA = P - A[x], PB = P - B[x], X = A[x] - B[x];
    d2 += X * X;
    os_1d(PA, PB, inv2p, la, lb, S[x]);
    double (*t)[8] = T[x];
    double (*o)[8] = S[x];
    t[0][0] = xi * (1.0 - 2.0 * xi * X * X);
    for (int i = 0; i < la; ++i) {
      double v = PA * t[i][0] + 2.0 * xi * o[i + 1][0];
      if (i > 0) v += i * inv2p * t[i - 1][0] - 2.0 * xi * (i / (2.0 * a1)) * o[i - 1][0];
      t[i + 1][0] = v;
    }
    for (int j = 0; j < lb; ++j)
      for (int i = 0; i <= la; ++i) {
        double v = PB * t[i][j] + 2.0 * xi * o[i][j + 1];
        if (i > 0) v += i * inv2p * t[i - 1][j];
        if (j > 0) v += j * inv2p * t[i][j - 1] - 2.0 * xi * (j / (2.0 * a2)) * o[i][j - 1];
        t[i][j + 1] = v;
      }
  }
  double pref = pow(ORC_PI / zeta, 1.5) * exp(-xi * d2);
  double pc[20][20];
  for (int p = 0; p < NCART[la]; ++p)
    for (int q = 0; q < NCART[lb]; ++q) {
      const int *u = CART[p], *w = CART[q];
      double sx = S[0][u[0]][w[0]], sy = S[1][u[1]][w[1]], sz = S[2][u[2]][w[2]];
      double tx = T[0][u[0]][w[0]], ty = T[1][u[1]][w[1]], tz = T[2][u[2]][w[2]];
      pc[p][q] = pref * (tx * sy * sz + sx * ty * sz + sx * sy * tz);
    }
  cart_to_sh(pc, la, lb, sh);
}

/* Mass-velocity integral (alpha^2 / 8) <a|nabla^4|b>, alpha the fine
 * structure constant 7.2973525693e-3 (constants.f90:47), the prefactor
 * (fineStructure * 0.001)^2 / 8 of gaussIntegrals.f90:39118.  The reference
 * builds it by a Cartesian recursion seeded with the s-s value
 * 16 a2^4 <r_B^4> - 80 a2^3 <r_B^2> + 60 a2^2 (nabla^4 on the atom-2
 * Gaussian).  Here it is the symmetric form <nabla^2 a|nabla^2 b>
 * (two integrations by parts), summed over axis pairs:
 *   sum_x U_x S_y S_z + sum_{x != y} L_x R_y S_z,
 * with the 1D second derivative d^2 x^i e^{-a x^2} = i(i-1) x^{i-2}
 * - 2a(2i+1) x^i + 4a^2 x^{i+2} applied on the left (L), the right (R) or
 * both (U) of the overlap table.  The s-s seed cancels to a value of order
 * a1 a2 when a1 << a2; the symmetric form carries that order in each term. */
static void d2_coef(int i, double a, double c[3]) {
  c[0] = i * (i - 1.0); /* x^{i-2} */
  c[1] = -2.0 * a * (2 * i + 1);
  c[2] = 4.0 * a * a;  /* x^{i+2} */
}

void orc_massvel2c(double a1, double a2, const double *A, const double *B,
                   int la, int lb, double *sh) {
  double zeta = a1 + a2, xi = a1 * a2 / zeta, d2 = 0.0;
  double S[3][8][8], L[3][4][4], R[3][4][4], U[3][4][4];
  for (int x = 0; x < 3; ++x) {
    double P = (a1 * A[x] + a2 * B[x]) / zeta;
    d2 += (A[x] - B[x]) * (A[x] - B[x]);
    os_1d(P - A[x], P - B[x], 1.0 / (2.0 * zeta), la + 2, lb + 2, S[x]);
    for (int i = 0; i <= la; ++i)
      for (int j = 0; j <= lb; ++j) {
        double ca[3], cb[3], l = 0.0, r = 0.0, u = 0.0;
        d2_coef(i, a1, ca);
        d2_coef(j, a2, cb);
        for (int p = 0; p < 3; ++p) {
          int ii = i + 2 * p - 2;
          if (ii < 0) continue;
          l += ca[p] * S[x][ii][j];
          for (int q = 0; q < 3; ++q) {
            int jj = j + 2 * q - 2;
            if (jj < 0) continue;
            u += ca[p] * cb[q] * S[x][ii][jj];
          }
        }
        for (int q = 0; q < 3; ++q) {
          int jj = j + 2 * q - 2;
          if (jj >= 0) r += cb[q] * S[x][i][jj];
        }
        L[x][i][j] = l;
        R[x][i][j] = r;
        U[x][i][j] = u;
      }
  }
  const double fs = 7.2973525693 * 0.001;
  double pref = fs * fs / 8.0 * pow(ORC_PI / zeta, 1.5) * exp(-xi * d2);
  double pc[20][20];
  for (int p = 0; p < NCART[la]; ++p)
    for (int q = 0; q < NCART[lb]; ++q) {
      const int *u = CART[p], *w = CART[q];
      double s[3], l[3], r[3], uu[3];
      for (int x = 0; x < 3; ++x) {
        s[x] = S[x][u[x]][w[x]];
        l[x] = L[x][u[x]][w[x]];
        r[x] = R[x][u[x]][w[x]];
        uu[x] = U[x][u[x]][w[x]];
      }
      double v = uu[0] * s[1] * s[2] + s[0] * uu[1] * s[2] + s[0] * s[1] * uu[2];
      v += (l[0] * r[1] + r[0] * l[1]) * s[2] + (l[0] * r[2] + r[0] * l[2]) * s[1] +
           (l[1] * r[2] + r[1] * l[2]) * s[0];
      pc[p][q] = pref * v;
    }
  cart_to_sh(pc, la, lb, sh);
}

/* Momentum and dipole blocks, three Cartesian components each (the
 * reference's sh(16,16,3)), sh3[c * 256 + i * 16 + j].  Both move the
 * operator into one 1D factor of the overlap table, the component's axis
 * taking the moved factor and the other two the plain overlap factors:
 *   dipole: (x - C_x) = x_B + (B_x - C_x) on atom 2's side;
 *   momentum: d/dx x^j e^{-a x^2} = j x^{j-1} - 2 a x^{j+1} on atom 2's
 *   side, or minus the same on atom 1's side (integration by parts), taken
 *   on the side of the smaller exponent: the overlap table's PB = P - B
 *   (PA = P - A) loses digits when P lies near B (near A), and the seed
 *   -2 a2 PB S = 2 a1 PA S is then formed from the other one.  The
 *   reference seeds with 2 a1 PA S (gaussIntegrals.f90:23080-23082). */
static void vec2c(int dipole, double a1, double a2, const double *A,
                  const double *B, const double *C, int la, int lb,
                  double *sh3) {
  double zeta = a1 + a2, xi = a1 * a2 / zeta, d2 = 0.0;
  double S[3][8][8], D[3][4][4];
  for (int x = 0; x < 3; ++x) {
    double P = (a1 * A[x] + a2 * B[x]) / zeta;
    d2 += (A[x] - B[x]) * (A[x] - B[x]);
    os_1d(P - A[x], P - B[x], 1.0 / (2.0 * zeta), la + 1, lb + 1, S[x]);
    for (int i = 0; i <= la; ++i)
      for (int j = 0; j <= lb; ++j) {
        if (dipole)
          D[x][i][j] = S[x][i][j + 1] + (B[x] - C[x]) * S[x][i][j];
        else if (a1 <= a2)
          D[x][i][j] = 2.0 * a1 * S[x][i + 1][j] - (i > 0 ? i * S[x][i - 1][j] : 0.0);
        else
          D[x][i][j] = -2.0 * a2 * S[x][i][j + 1] + (j > 0 ? j * S[x][i][j - 1] : 0.0);
      }
  }
  double pref = pow(ORC_PI / zeta, 1.5) * exp(-xi * d2);
  double pc[20][20];
  for (int c = 0; c < 3; ++c) {
    for (int p = 0; p < NCART[la]; ++p)
      for (int q = 0; q < NCART[lb]; ++q) {
        const int *u = CART[p], *w = CART[q];
        double v = 1.0;
        for (int x = 0; x < 3; ++x)
          v *= (x == c) ? D[x][u[x]][w[x]] : S[x][u[x]][w[x]];
        pc[p][q] = pref * v;
      }
    cart_to_sh(pc, la, lb, sh3 + 256 * c);
  }
}

void orc_momentum2c(double a1, double a2, const double *A, const double *B,
                    int la, int lb, double *sh3) {
  vec2c(0, a1, a2, A, B, NULL, la, lb, sh3);
}

void orc_dipole2c(double a1, double a2, const double *A, const double *B,
                  const double *C, int la, int lb, double *sh3) {
  vec2c(1, a1, a2, A, B, C, la, lb, sh3);
}

/* Overlap with a plane wave, <a|exp(-i dK.r)|b> (complex).  The product
 * Gaussian times exp(-i q x) is exp(-i q P - q^2/(4p)) times a Gaussian
 * about P' = P - i q/(2p), so the 1D recursion runs with the complex
 * PA' = PA - i q/(2p), PB' = PB - i q/(2p) and each axis carries
 * sqrt(pi/p) exp(-xi X^2) exp(-q^2/(4p)) exp(-i q P).  The reference
 * writes the same shift as Hermite-polynomial terms (hermite_term(1) =
 * -i q/(2p); hermite_term(2) - hermite_term(1)^2 = 1/(2p),
 * gaussIntegrals.f90:129450-129470).  sh2[2 * (i*16 + j) + 0/1] = re/im. */
void orc_koverlap2c(double a1, double a2, const double *A, const double *B,
                    const double *dK, int la, int lb, double *sh2) {
  const double zeta = a1 + a2, xi = a1 * a2 / zeta, inv2p = 1.0 / (2.0 * zeta);
  double Sr[3][8][8], Si[3][8][8], pr[3], pi_[3];
  for (int x = 0; x < 3; ++x) {
    const double P = (a1 * A[x] + a2 * B[x]) / zeta, X = A[x] - B[x];
    const double ar = P - A[x], br = P - B[x], sh = -dK[x] * inv2p;  /* imag shift */
    /* S_{i+1,j} = PA' S_ij + (i S_{i-1,j} + j S_{i,j-1}) / (2p), complex */
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
    const double mag = sqrt(ORC_PI / zeta) * exp(-xi * X * X) *
                       exp(-dK[x] * dK[x] / (4.0 * zeta));
    pr[x] = mag * cos(dK[x] * P);
    pi_[x] = -mag * sin(dK[x] * P);
  }
  double pcr[20][20], pci[20][20];
  for (int p = 0; p < NCART[la]; ++p)
    for (int q = 0; q < NCART[lb]; ++q) {
      double vr = 1.0, vi = 0.0;
      for (int x = 0; x < 3; ++x) {
        const int i = CART[p][x], j = CART[q][x];
        /* times S_x(i, j) * pref_x */
        const double fr = Sr[x][i][j] * pr[x] - Si[x][i][j] * pi_[x];
        const double fi = Sr[x][i][j] * pi_[x] + Si[x][i][j] * pr[x];
        const double nr = vr * fr - vi * fi, ni = vr * fi + vi * fr;
        vr = nr;
        vi = ni;
      }
      pcr[p][q] = vr;
      pci[p][q] = vi;
    }
  double shr[256], shi[256];
  cart_to_sh(pcr, la, lb, shr);
  cart_to_sh(pci, la, lb, shi);
  for (int k = 0; k < 256; ++k) {
    sh2[2 * k] = shr[k];
    sh2[2 * k + 1] = shi[k];
  }
}

/* Three-centre overlap: the three Gaussians combine into one of exponent
 * zeta3 = a1 + a2 + a3 centred at G, and the 1D recursion runs about G. */
void orc_electron3c(double a1, double a2, double a3, const double *A,
                    const double *B, const double *C, int la, int lb,
                    double *sh) {
  double zeta = a1 + a2, zeta3 = zeta + a3, xi = a1 * a2 / zeta;
  double d2 = 0.0, pc2 = 0.0;
  double S[3][8][8];
  for (int x = 0; x < 3; ++x) {
    double P = (a1 * A[x] + a2 * B[x]) / zeta;
    double G = (a1 * A[x] + a2 * B[x] + a3 * C[x]) / zeta3;
    d2 += (A[x] - B[x]) * (A[x] - B[x]);
    pc2 += (P - C[x]) * (P - C[x]);
    os_1d(G - A[x], G - B[x], 1.0 / (2.0 * zeta3), la, lb, S[x]);
  }
  double pref = pow(ORC_PI / zeta3, 1.5) *
                exp(-xi * d2 - (zeta * a3 / zeta3) * pc2);
  double pc[20][20];
  for (int p = 0; p < NCART[la]; ++p)
    for (int q = 0; q < NCART[lb]; ++q)
      pc[p][q] = pref * S[0][CART[p][0]][CART[q][0]] *
                 S[1][CART[p][1]][CART[q][1]] * S[2][CART[p][2]][CART[q][2]];
  cart_to_sh(pc, la, lb, sh);
}

/* Three-centre nuclear integral.  Vertical recursion on the atom-1 index
 * with auxiliary order m,
 *   (e+1_i|0)^m = GA_i (e|0)^m - GC_i (e|0)^{m+1}
 *                 + e_i/(2 zeta3) [(e-1_i|0)^m - (e-1_i|0)^{m+1}],
 *   (0|0)^m = 2 pi / zeta3 * K * F_m(zeta3 |G-C|^2),
 * then the atom-2 index is moved over with x_B = x_A + (A-B):
 *   (a|b) = sum_k prod_axes C(b,k) (A-B)^{b-k} (a+k|0). */
void orc_nuclear3c(double a1, double a2, double a3, const double *A,
                   const double *B, const double *C, int la, int lb,
                   double *sh) {
  double zeta = a1 + a2, zeta3 = zeta + a3;
  double G[3], GA[3], GC[3], AB[3];
  double U = 0.0, ex = 0.0;
  for (int x = 0; x < 3; ++x) {
    G[x] = (a1 * A[x] + a2 * B[x] + a3 * C[x]) / zeta3;
    GA[x] = G[x] - A[x];
    GC[x] = G[x] - C[x];
    AB[x] = A[x] - B[x];
    U += GC[x] * GC[x];
    double d1 = A[x] - B[x], dd2 = A[x] - C[x], d3 = B[x] - C[x];
    ex += a1 * a2 * d1 * d1 + a1 * a3 * dd2 * dd2 + a2 * a3 * d3 * d3;
  }
  U *= zeta3;
  double F[7];
  orc_boys(U, F);
  const int L = la + lb;
  double K = 2.0 * (ORC_PI / zeta3) * exp(-ex / zeta3);
  /* V[m][ex][ey][ez] for ex+ey+ez <= L, m <= L - (ex+ey+ez). */
  double V[7][7][7][7];
  for (int m = 0; m <= L; ++m) V[m][0][0][0] = F[m] * K;
  double inv2z3 = 1.0 / (2.0 * zeta3);
  for (int n = 1; n <= L; ++n)
    for (int e0 = n; e0 >= 0; --e0)
      for (int e1 = n - e0; e1 >= 0; --e1) {
        int e2 = n - e0 - e1;
        int e[3] = {e0, e1, e2};
        int ax = e0 > 0 ? 0 : (e1 > 0 ? 1 : 2);
        int p[3] = {e0, e1, e2};
        p[ax] -= 1;
        for (int m = 0; m <= L - n; ++m) {
          double v = GA[ax] * V[m][p[0]][p[1]][p[2]] -
                     GC[ax] * V[m + 1][p[0]][p[1]][p[2]];
          if (p[ax] > 0) {
            int q[3] = {p[0], p[1], p[2]};
            q[ax] -= 1;
            v += p[ax] * inv2z3 *
                 (V[m][q[0]][q[1]][q[2]] - V[m + 1][q[0]][q[1]][q[2]]);
          }
          V[m][e[0]][e[1]][e[2]] = v;
        }
      }
  static const double BIN[4][4] = {
      {1, 0, 0, 0}, {1, 1, 0, 0}, {1, 2, 1, 0}, {1, 3, 3, 1}};
  double pc[20][20];
  for (int p = 0; p < NCART[la]; ++p)
    for (int q = 0; q < NCART[lb]; ++q) {
      const int *a = CART[p], *b = CART[q];
      double s = 0.0;
      for (int kx = 0; kx <= b[0]; ++kx)
        for (int ky = 0; ky <= b[1]; ++ky)
          for (int kz = 0; kz <= b[2]; ++kz) {
            double w = BIN[b[0]][kx] * BIN[b[1]][ky] * BIN[b[2]][kz] *
                       pow(AB[0], b[0] - kx) * pow(AB[1], b[1] - ky) *
                       pow(AB[2], b[2] - kz);
            s += w * V[0][a[0] + kx][a[1] + ky][a[2] + kz];
          }
      pc[p][q] = s;
    }
  cart_to_sh(pc, la, lb, sh);
}
