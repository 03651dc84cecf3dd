// k_eval.cu -- single primitive integrals for checking the device
// arithmetic against the reference's generated kernels.
#include "intg.cuh"
#include "prim.cuh"

namespace imago {

// ---------------------------------------------------------- prim_eval --
// Single primitives for checking against the reference's kernels.
template <int LA, int LB>
__device__ void eval_one(int kind, const double *p, double *out) {
  constexpr int L = LA + LB;
  const double a1 = p[0], a2 = p[1], a3 = p[2];
  const double *A = p + 3, *B = p + 6, *C = p + 9;
  double blk[nsh(LA) * nsh(LB)];
  if (kind == 0) {
    prim2c<LA, LB, false>(a1, a2, A, B, blk);
  } else if (kind == 1) {
    prim2c<LA, LB, true>(a1, a2, A, B, blk);
  } else {
    const double zeta = a1 + a2, xi = a1 * a2 / zeta, z3 = zeta + a3;
    double X[3], d2 = 0.0;
#pragma unroll
    for (int x = 0; x < 3; ++x) {
      X[x] = (a1 * A[x] + a2 * B[x]) / zeta - C[x];
      d2 += (A[x] - B[x]) * (A[x] - B[x]);
    }
    double Q[nherm(L)];
#pragma unroll
    for (int i = 0; i < nherm(L); ++i) Q[i] = 0.0;
    double pref;
    if (kind == 2) {
      accumulate_overlap_q<L>(X, zeta * a3 / z3, 1.0, Q);
      pref = pow(kPi / z3, 1.5) * exp(-xi * d2);
    } else {
      accumulate_nuclear_q<L>(X, zeta * a3 / z3, zeta * zeta / z3,
                              2.0 * kPi / z3, Q);
      pref = exp(-xi * d2);
    }
    hermite_to_sh<LA, LB>(A, B, a1, a2, pref, Q, blk);
  }
  for (int i = 0; i < 256; ++i) out[i] = 0.0;
  for (int i = 0; i < nsh(LA); ++i)
    for (int j = 0; j < nsh(LB); ++j) out[i * 16 + j] = blk[i * nsh(LB) + j];
}

template <int LA, int LB>
__device__ void eval_mv(const double *p, double *out) {
  double blk[nsh(LA) * nsh(LB)];
  prim_mv<LA, LB>(p[0], p[1], p + 3, p + 6, kMassVelPref, blk);
  for (int i = 0; i < 256; ++i) out[i] = 0.0;
  for (int i = 0; i < nsh(LA); ++i)
    for (int j = 0; j < nsh(LB); ++j) out[i * 16 + j] = blk[i * nsh(LB) + j];
}

// One component of the momentum (DIP = false) or dipole blocks (the
// dipole centre is params 9..11), every class through the runtime-class
// routine: the build kernels' unrolled s/p/d variants share its arithmetic
// (vec_factor, the same tables) and are checked by the build tests.
template <bool DIP>
__device__ void eval_vec_rt(int la, int lb, int comp, const double *p, double *out) {
  const int nb = nsh(la) * nsh(lb);
  double blk[3 * 256];
  prim_vec_rt<DIP>(la, lb, p[0], p[1], p + 3, p + 6, p + 9, blk, nb);
  for (int i = 0; i < 256; ++i) out[i] = 0.0;
  for (int i = 0; i < nsh(la); ++i)
    for (int j = 0; j < nsh(lb); ++j) out[i * 16 + j] = blk[comp * nb + i * nsh(lb) + j];
}

static __device__ void eval_one_rt(int la, int lb, int kind, const double *p,
                            double *out) {
  const int L = la + lb;
  const double a1 = p[0], a2 = p[1], a3 = p[2];
  const double *A = p + 3, *B = p + 6, *C = p + 9;
  double blk[256];
  if (kind == 0 || kind == 1) {
    prim2c_rt(la, lb, kind == 1, a1, a2, A, B, blk);
  } else {
    const double zeta = a1 + a2, xi = a1 * a2 / zeta, z3 = zeta + a3;
    double X[3], d2 = 0.0;
    for (int x = 0; x < 3; ++x) {
      X[x] = (a1 * A[x] + a2 * B[x]) / zeta - C[x];
      d2 += (A[x] - B[x]) * (A[x] - B[x]);
    }
    double Q[kMaxHerm];
    for (int i = 0; i < kMaxHerm; ++i) Q[i] = 0.0;
    double pref;
    if (kind == 2) {
      accumulate_overlap_q_rt(L, X, zeta * a3 / z3, 1.0, Q);
      pref = pow(kPi / z3, 1.5) * exp(-xi * d2);
    } else {
      accumulate_nuclear_q_rt(L, X, zeta * a3 / z3, zeta * zeta / z3,
                              2.0 * kPi / z3, Q);
      pref = exp(-xi * d2);
    }
    hermite_to_sh_rt(la, lb, A, B, a1, a2, pref, Q, blk);
  }
  for (int i = 0; i < 256; ++i) out[i] = 0.0;
  for (int i = 0; i < nsh(la); ++i)
    for (int j = 0; j < nsh(lb); ++j) out[i * 16 + j] = blk[i * nsh(lb) + j];
}

__global__ void k_prim_eval(int kind, int n, const double *params,
                            const int *cls, double *sh) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const double *p = params + 12 * r;
  double *out = sh + 256 * (long long)r;
  if (kind == 4) {
    double F[7];
    boys_ref<6>(p[0], F);
    for (int i = 0; i < 256; ++i) out[i] = 0.0;
    for (int i = 0; i < 7; ++i) out[i] = F[i];
    return;
  }
  const int la = cls[2 * r], lb = cls[2 * r + 1];
  if (kind >= 6) {  // momentum (6..8) / dipole (9..11), components x, y, z
    const int comp = (kind - 6) % 3;
    const bool dip = kind >= 9;
    if (dip)
      eval_vec_rt<true>(la, lb, comp, p, out);
    else
      eval_vec_rt<false>(la, lb, comp, p, out);
    return;
  }
  if (kind == 5) {  // mass velocity: s/p/d unrolled, f at run time
    switch (la * 4 + lb) {
#define IMAGO_EV(a, b) \
  case a * 4 + b:      \
    eval_mv<a, b>(p, out); \
    break;
      IMAGO_EV(0, 0) IMAGO_EV(0, 1) IMAGO_EV(0, 2) IMAGO_EV(1, 0)
      IMAGO_EV(1, 1) IMAGO_EV(1, 2) IMAGO_EV(2, 0) IMAGO_EV(2, 1)
      IMAGO_EV(2, 2)
#undef IMAGO_EV
      default: {
        double blk[256];
        prim_mv_rt(la, lb, p[0], p[1], p + 3, p + 6, kMassVelPref, blk);
        for (int i = 0; i < 256; ++i) out[i] = 0.0;
        for (int i = 0; i < nsh(la); ++i)
          for (int j = 0; j < nsh(lb); ++j) out[i * 16 + j] = blk[i * nsh(lb) + j];
        break;
      }
    }
    return;
  }
  switch (la * 4 + lb) {
#define IMAGO_EV(a, b) \
  case a * 4 + b:      \
    eval_one<a, b>(kind, p, out); \
    break;
    IMAGO_EV(0, 0) IMAGO_EV(0, 1) IMAGO_EV(0, 2) IMAGO_EV(1, 0) IMAGO_EV(1, 1)
    IMAGO_EV(1, 2) IMAGO_EV(2, 0) IMAGO_EV(2, 1) IMAGO_EV(2, 2)
#undef IMAGO_EV
    default:
      eval_one_rt(la, lb, kind, p, out);
      break;
  }
}

int launch_prim_eval(int kind, int n, const double *params, const int *cls,
                     double *sh, cudaStream_t st) {
  if (n <= 0) return IMAGO_OK;
  k_prim_eval<<<(n + 63) / 64, 64, 0, st>>>(kind, n, params, cls, sh);
  IMAGO_CUDA(cudaGetLastError());
  return IMAGO_OK;
}

}  // namespace imago
