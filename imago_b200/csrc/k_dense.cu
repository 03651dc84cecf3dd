// k_dense.cu -- contraction, lattice-to-k phase sums, scatter and core
// orthogonalisation of one integral build.
#include "intg.cuh"

namespace imago {

// ---------------------------------------------------------- contract --
// One warp per (unit, term):
//   M(m1, m2) = sum_{(a,b) in unit} C1(a, m1) C2(b, m2) sh_ab(lm1, lm2),
// the pairXBasisFn2 / multWithBasisFn1 contraction (integrals.F90:555-563,
// intgSaving.F90:56-89).  Terms with lm beyond a primitive's class carry a
// zero coefficient in the reference and are skipped here.
__global__ void __launch_bounds__(256)
    k_contract(DevSys s, DevWork w, int nterm, const double *blk, double *M) {
  const long long wid =
      ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (wid >= (long long)w.nunits * nterm) return;
  const int term = (int)(wid / w.nunits);
  const int ui = (int)(wid % w.nunits);
  const DUnit u = w.units[ui];
  const DPair p = w.pairs[u.pair];
  const int ni = p.ni, nj = p.nj, ne = ni * nj;
  const double *bk = blk + (long long)term * w.blk_total;
  double *out = M + (long long)term * w.m_total + p.moff +
                (long long)(ui - p.ubeg) * ne;
  const int so1 = s.type_state_off[p.ti], so2 = s.type_state_off[p.tj];
  const double *c1 = s.basis + s.type_basis_off[p.ti];
  const double *c2 = s.basis + s.type_basis_off[p.tj];
  for (int e = lane; e < ne; e += 32) {
    const int m1 = e / nj, m2 = e - m1 * nj;
    const int lm1 = s.state_lm[so1 + m1], lm2 = s.state_lm[so2 + m2];
    double acc = 0.0;
    for (int q = u.spbeg; q < u.spend; ++q) {
      const DSp sp = w.sps[q];
      const int na = nsh(sp.la), nb = nsh(sp.lb);
      if (lm1 >= na || lm2 >= nb) continue;
      acc += c1[sp.a * ni + m1] * c2[sp.b * nj + m2] *
             bk[sp.boff + lm1 * nb + lm2];
    }
    out[e] = acc;
  }
}

int launch_contract(const DevSys &s, const DevWork &w, int nterm,
                    const double *blk, double *M, cudaStream_t st) {
  const long long warps = (long long)w.nunits * nterm;
  if (warps == 0) return IMAGO_OK;
  const int tb = 256;
  const long long grid = (warps * 32 + tb - 1) / tb;
  k_contract<<<(unsigned)grid, tb, 0, st>>>(s, w, nterm, blk, M);
  IMAGO_CUDA(cudaGetLastError());
  return IMAGO_OK;
}

// ------------------------------------------------------------- bloch --
// P_pair(k) = exp(i k.L0) sum_{images} exp(i k.R) M(R), then the block is
// scattered as saveCurrentPair does (valence first, core after, dagger for
// the transposed core blocks, the last write winning for i == j).
constexpr int kBlochK = 16;

__device__ __forceinline__ void scatter(const DevSys &s, const DPair &p,
                                        int term, int k, int m1, int m2,
                                        double re, double im, double2 *vv,
                                        double2 *cv, double2 *cc) {
  const int V = s.vale_dim, C = s.core_dim;
  const int v1 = s.type_nvale[p.ti], v2 = s.type_nvale[p.tj];
  const long long tk = (long long)term * s.nk + k;
  if (m1 < v1 && m2 < v2) {
    if (p.i == p.j && m1 > m2) return;  // lower triangle: never read
    const int row = s.site_cum_vale[p.i] + m1, col = s.site_cum_vale[p.j] + m2;
    vv[tk * V * V + (long long)col * V + row] = make_double2(re, im);
    return;
  }
  if (C == 0) return;
  if (m1 >= v1 && m2 < v2) {
    if (p.i == p.j) return;  // overwritten by the dagger block
    const int row = s.site_cum_core[p.i] + (m1 - v1);
    const int col = s.site_cum_vale[p.j] + m2;
    cv[tk * V * C + (long long)col * C + row] = make_double2(re, im);
  } else if (m1 < v1) {
    const int row = s.site_cum_core[p.j] + (m2 - v2);
    const int col = s.site_cum_vale[p.i] + m1;
    cv[tk * V * C + (long long)col * C + row] = make_double2(re, -im);
  } else {
    const int r1 = s.site_cum_core[p.i] + (m1 - v1);
    const int r2 = s.site_cum_core[p.j] + (m2 - v2);
    cc[tk * C * C + (long long)r2 * C + r1] = make_double2(re, im);
    if (p.i != p.j)
      cc[tk * C * C + (long long)r1 * C + r2] = make_double2(re, -im);
  }
}

__global__ void __launch_bounds__(128)
    k_bloch(DevSys s, DevWork w, const double *M, double2 *vv, double2 *cv,
            double2 *cc) {
  const int pi = blockIdx.x, term = blockIdx.y, k0 = blockIdx.z * kBlochK;
  const DPair p = w.pairs[pi];
  const int ne = p.ni * p.nj;
  const double *Mt = M + (long long)term * w.m_total + p.moff;
  const int nk = s.nk;
  double cs[kBlochK], sn[kBlochK];
#pragma unroll
  for (int kk = 0; kk < kBlochK; ++kk) {
    cs[kk] = 1.0;
    sn[kk] = 0.0;
    const int k = k0 + kk;
    if (k < nk) {
      const double *kv = s.kxyz + 3 * k;
      const double dot = kv[0] * p.L0[0] + kv[1] * p.L0[1] + kv[2] * p.L0[2];
      // kPointLatticeOriginShift (intgSaving.F90:241-292) skips the shift
      // when |k.L0| < smallThresh.
      if (fabs(dot) >= kSmallThresh) sincos(dot, &sn[kk], &cs[kk]);
    }
  }
  for (int e = threadIdx.x; e < ne; e += blockDim.x) {
    double re[kBlochK], im[kBlochK];
#pragma unroll
    for (int kk = 0; kk < kBlochK; ++kk) re[kk] = im[kk] = 0.0;
    for (int u = p.ubeg; u < p.uend; ++u) {
      const double x = Mt[(long long)(u - p.ubeg) * ne + e];
      const double2 *ph = s.phase + (long long)w.units[u].cell * nk + k0;
#pragma unroll
      for (int kk = 0; kk < kBlochK; ++kk)
        if (k0 + kk < nk) {
          const double2 f = ph[kk];
          re[kk] += f.x * x;
          im[kk] += f.y * x;
        }
    }
    const int m1 = e / p.nj, m2 = e - m1 * p.nj;
#pragma unroll
    for (int kk = 0; kk < kBlochK; ++kk) {
      const int k = k0 + kk;
      if (k >= nk) break;
      const double r = cs[kk] * re[kk] - sn[kk] * im[kk];
      const double i = cs[kk] * im[kk] + sn[kk] * re[kk];
      scatter(s, p, term, k, m1, m2, r, i, vv, cv, cc);
    }
  }
}

int launch_bloch(const DevSys &s, const DevWork &w, int nterm, const double *M,
                 double2 *vv, double2 *cv, double2 *cc, cudaStream_t st) {
  if (w.npairs == 0 || nterm == 0) return IMAGO_OK;
  dim3 grid(w.npairs, nterm, (s.nk + kBlochK - 1) / kBlochK);
  k_bloch<<<grid, 128, 0, st>>>(s, w, M, vv, cv, cc);
  IMAGO_CUDA(cudaGetLastError());
  return IMAGO_OK;
}

// ------------------------------------------------------------- ortho --
// With S = coreValeOL and X the matrix being orthogonalised, the reference
// computes (zherk or zher2k on the upper triangle, then coreValeCoreCore
// and makeValeVale):
//   VV' = VV - S^H X_cv - X_cv^H S + S^H X_cc S.
// Here the same is formed as VV' = VV - (S^H Y + Y^H S) with
// Y = X_cv - X_cc S / 2, which needs one product less (X_cc is Hermitian).
// For the overlap itself X = S and this is VV - 2 S^H S + S^H S_cc S.
__global__ void __launch_bounds__(256)
    k_ortho_y(DevSys s, const double2 *cv, const double2 *cc,
              const double2 *s_cv, double2 *y) {
  const int k = blockIdx.y, term = blockIdx.z;
  const int V = s.vale_dim, C = s.core_dim;
  const long long tk = (long long)term * s.nk + k;
  const double2 *X = cv + tk * V * C;
  const double2 *XC = cc + tk * C * C;
  const double2 *S = s_cv + (long long)k * V * C;
  double2 *Y = y + tk * V * C;
  const long long n = (long long)V * C;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
       idx < n; idx += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(idx % C), v = (int)(idx / C);
    double ar = 0.0, ai = 0.0;
    for (int l = 0; l < C; ++l) {
      const double2 a = XC[(long long)l * C + c];  // X_cc(c, l)
      const double2 b = S[(long long)v * C + l];   // S(l, v)
      ar += a.x * b.x - a.y * b.y;
      ai += a.x * b.y + a.y * b.x;
    }
    const double2 x = X[idx];
    Y[idx] = make_double2(x.x - 0.5 * ar, x.y - 0.5 * ai);
  }
}

__global__ void __launch_bounds__(256)
    k_ortho_pack(DevSys s, const double2 *vv, const double2 *y,
                 const double2 *s_cv, double *packed) {
  const int k = blockIdx.y, term = blockIdx.z;
  const int V = s.vale_dim, C = s.core_dim;
  const long long np = (long long)V * (V + 1) / 2;
  const long long tk = (long long)term * s.nk + k;
  const double2 *VVt = vv + tk * V * V;
  const double2 *Y = y + tk * V * C;
  const double2 *S = s_cv + (long long)k * V * C;
  double *out = packed + 2 * tk * np;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
       idx < np; idx += (long long)gridDim.x * blockDim.x) {
    int col = (int)((sqrt(8.0 * (double)idx + 1.0) - 1.0) * 0.5);
    while ((long long)col * (col + 1) / 2 > idx) --col;
    while ((long long)(col + 1) * (col + 2) / 2 <= idx) ++col;
    const int row = (int)(idx - (long long)col * (col + 1) / 2);
    double2 v = VVt[(long long)col * V + row];
    if (C > 0) {
      double sr = 0.0, si = 0.0;
      const double2 *Sr = S + (long long)row * C, *Sc = S + (long long)col * C;
      const double2 *Yr = Y + (long long)row * C, *Yc = Y + (long long)col * C;
      for (int l = 0; l < C; ++l) {
        const double2 a = Sr[l], b = Yc[l], c = Yr[l], d = Sc[l];
        // conj(a) b + conj(c) d
        sr += a.x * b.x + a.y * b.y + c.x * d.x + c.y * d.y;
        si += a.x * b.y - a.y * b.x + c.x * d.y - c.y * d.x;
      }
      v.x -= sr;
      v.y -= si;
      if (row == col) v.y = 0.0;  // zherk/zher2k keep the diagonal real
      if (fabs(v.x) < kPackThresh) v.x = 0.0;
      if (fabs(v.y) < kPackThresh) v.y = 0.0;
    }
    out[2 * idx] = v.x;
    out[2 * idx + 1] = v.y;
  }
}

int launch_ortho(const DevSys &s, int nterm, const double2 *vv,
                 const double2 *cv, const double2 *cc, const double2 *s_cv,
                 double2 *y, double *packed, cudaStream_t st) {
  const int V = s.vale_dim, C = s.core_dim;
  if (nterm == 0) return IMAGO_OK;
  if (C > 0) {
    const long long n = (long long)V * C;
    dim3 g((unsigned)((n + 255) / 256 > 64 ? 64 : (n + 255) / 256), s.nk, nterm);
    k_ortho_y<<<g, 256, 0, st>>>(s, cv, cc, s_cv, y);
    IMAGO_CUDA(cudaGetLastError());
  }
  const long long np = (long long)V * (V + 1) / 2;
  dim3 g2((unsigned)((np + 255) / 256 > 128 ? 128 : (np + 255) / 256), s.nk, nterm);
  k_ortho_pack<<<g2, 256, 0, st>>>(s, vv, y, s_cv, packed);
  IMAGO_CUDA(cudaGetLastError());
  return IMAGO_OK;
}

// coreValeOL as the reference writes it: separate real and imaginary
// (coreDim, valeDim) matrices per k.
__global__ void k_split_cv(long long n, const double2 *cv, double *re,
                           double *im) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double2 v = cv[i];
    re[i] = v.x;
    im[i] = v.y;
  }
}

int launch_split_cv(const DevSys &s, const double2 *cv, double *re, double *im,
                    cudaStream_t st) {
  const long long n = (long long)s.nk * s.vale_dim * s.core_dim;
  if (n == 0) return IMAGO_OK;
  k_split_cv<<<(unsigned)((n + 255) / 256 > 4096 ? 4096 : (n + 255) / 256), 256, 0, st>>>(
      n, cv, re, im);
  IMAGO_CUDA(cudaGetLastError());
  return IMAGO_OK;
}

// phaseFactor(k, cell) = exp(i k.R) (kpoints.f90:578-609), stored cell-major
// so one image's phases for consecutive k are contiguous.
__global__ void k_phase(DevSys s, double2 *phase) {
  const long long n = (long long)s.ncell * s.nk;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i / s.nk), k = (int)(i % s.nk);
    const double *kv = s.kxyz + 3 * k, *R = s.cell + 3 * c;
    const double dot = kv[0] * R[0] + kv[1] * R[1] + kv[2] * R[2];
    double sn, cs;
    sincos(dot, &sn, &cs);
    phase[i] = make_double2(cs, sn);
  }
}

int launch_phase(const DevSys &s, double2 *phase, cudaStream_t st) {
  const long long n = (long long)s.ncell * s.nk;
  k_phase<<<(unsigned)((n + 255) / 256 > 4096 ? 4096 : (n + 255) / 256), 256, 0, st>>>(s, phase);
  IMAGO_CUDA(cudaGetLastError());
  return IMAGO_OK;
}

}  // namespace imago
