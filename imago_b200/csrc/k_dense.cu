// k_dense.cu -- contraction, lattice-to-k phase sums, scatter and core
// orthogonalisation of one integral build.
//
// The phase sums and the orthogonalisation are dense complex contractions
// and run on the FP64 tensor cores (mma.sync m8n8k4 f64), tiled through
// shared memory.
#include <algorithm>

#include "intg.cuh"
#include "tma.cuh"

namespace imago {

// D += A * B for one 8x8x4 FP64 tile.  Fragments (PTX ISA, mma.m8n8k4 .f64):
// a = A(row = lane/4, k = lane%4), b = B(k = lane%4, col = lane/4),
// d[i] = D(row = lane/4, col = 2*(lane%4) + i).
__device__ __forceinline__ void dmma(double &d0, double &d1, double a,
                                     double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, "
      "{%0,%1};"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

// One packed (re, im) element: a single 16-byte store when the caller's
// buffer allows it (device allocations do), two 8-byte stores otherwise.
__device__ __forceinline__ void store_packed(double *out, long long idx, double2 v) {
  if (((size_t)out & 15) == 0)
    reinterpret_cast<double2 *>(out)[idx] = v;
  else {
    out[2 * idx] = v.x;
    out[2 * idx + 1] = v.y;
  }
}

// 16-byte global-to-shared copy that does not pass through registers;
// with `valid` false nothing is read and the destination is zero-filled.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem,
                                           bool valid) {
  const unsigned dst = (unsigned)__cvta_generic_to_shared(smem);
  const int n = valid ? 16 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst),
               "l"(gmem), "r"(n)
               : "memory");
}

// 8-byte copy with zero fill when `valid` is false (nothing is read).
__device__ __forceinline__ void cp_async8z(void *smem, const void *gmem,
                                           bool valid) {
  const unsigned dst = (unsigned)__cvta_generic_to_shared(smem);
  const int n = valid ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst),
               "l"(gmem), "r"(n)
               : "memory");
}

// 8-byte global-to-shared copy that does not pass through registers.
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
  const unsigned dst = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(gmem)
               : "memory");
}

// ---------------------------------------------------------- contract --
// One CTA per (unit, group of terms), threads over the block elements:
//   M_t(m1, m2) = sum_{(a,b) in unit} C1(a, m1) C2(b, m2) sh_t,ab(lm1, lm2),
// the pairXBasisFn2 / multWithBasisFn1 contraction (integrals.F90:555-563,
// intgSaving.F90:56-89).  Entries whose lm lies beyond a primitive's class
// carry a zero coefficient in the reference and are skipped.  Blocks are
// stored column-major, e = m2 * ni + m1.  A unit's primitive blocks of one
// term are contiguous in `blk`: they are staged through shared memory in
// chunks of whole shell pairs with coalesced loads, together with the
// chunk's shell-pair list and both atoms' coefficient tables; the
// coefficient product of an (element, shell pair) serves every term of
// the group.  T = 4 or 8 terms per CTA, picked by measurement: eight halve
// the per-(element, shell pair) work of a many-term build but give fewer
// CTAs and a smaller staging chunk.
constexpr int kContractThreads = 128;
constexpr int kElemsPerThread = 3;          // n_i n_j <= 384 per pass
constexpr int kSpStage = 256;               // shell pairs staged at a time
constexpr int kCoefMax = 1024;              // alphas x states per atom

template <int T>
__global__ void __launch_bounds__(kContractThreads, 4)
    k_contract(DevSys s, DevWork w, int nterm, const double *blk, double *M) {
  constexpr int kTermsPerCta = T;
  constexpr int kBlkStage = T >= 8 ? 384 : 768;  // block doubles per term staged
  __shared__ int sp_ab[kSpStage];            // a | b << 16
  __shared__ int sp_cls[kSpStage];           // nsh(la) | nsh(lb) << 8
  __shared__ int sp_rel[kSpStage];           // block offset from the chunk's
  __shared__ double c1s[kCoefMax], c2s[kCoefMax];
  __shared__ double bs[kTermsPerCta][kBlkStage];
  __shared__ long long chunk_base;
  const int ntg = (nterm + kTermsPerCta - 1) / kTermsPerCta;
  const int ui = blockIdx.x / ntg;
  const int t0 = (blockIdx.x % ntg) * kTermsPerCta;
  const int tn = min(kTermsPerCta, nterm - t0);
  const int tid = threadIdx.x;
  const DUnit u = w.units[ui];
  const DPair p = w.pairs[u.pair];
  const int ni = p.ni, nj = p.nj, ne = ni * nj;
  const int na1 = s.type_nalpha[p.ti], na2 = s.type_nalpha[p.tj];
  const long long base = p.moff + (long long)(ui - p.ubeg) * ne;
  const int so1 = s.type_state_off[p.ti], so2 = s.type_state_off[p.tj];
  const double *c1 = s.basis + s.type_basis_off[p.ti];
  const double *c2 = s.basis + s.type_basis_off[p.tj];
  const bool stage_coef = na1 * ni <= kCoefMax && na2 * nj <= kCoefMax;
  if (stage_coef) {
    for (int i = tid; i < na1 * ni; i += kContractThreads) c1s[i] = c1[i];
    for (int i = tid; i < na2 * nj; i += kContractThreads) c2s[i] = c2[i];
  }
  const double *cf1 = stage_coef ? c1s : c1;
  const double *cf2 = stage_coef ? c2s : c2;
  const double *bt = blk + (long long)t0 * w.blk_total;
  for (int e0 = 0; e0 < ne; e0 += kContractThreads * kElemsPerThread) {
    int lm1[kElemsPerThread], lm2[kElemsPerThread], m1[kElemsPerThread],
        m2[kElemsPerThread];
    double acc[kElemsPerThread][kTermsPerCta];
#pragma unroll
    for (int j = 0; j < kElemsPerThread; ++j) {
      const int e = e0 + tid + j * kContractThreads;
      m2[j] = e < ne ? e / ni : 0;
      m1[j] = e < ne ? e - m2[j] * ni : 0;
      lm1[j] = e < ne ? s.state_lm[so1 + m1[j]] : 1 << 20;
      lm2[j] = e < ne ? s.state_lm[so2 + m2[j]] : 1 << 20;
#pragma unroll
      for (int t = 0; t < kTermsPerCta; ++t) acc[j][t] = 0.0;
    }
    for (int q0 = u.spbeg; q0 < u.spend;) {
      const int nq = min(kSpStage, u.spend - q0);
      __syncthreads();
      // shell pairs of the chunk: those whose blocks end within kBlkStage
      // doubles of the first one's start (at least one: a block has <= 256)
      int fit = 0;
      for (int i = tid; i < kSpStage; i += kContractThreads) {
        if (i < nq) {
          const DSp sp = w.sps[q0 + i];
          const long long b0 = w.sps[q0].boff;
          const int rel = (int)(sp.boff - b0);
          sp_ab[i] = sp.a | (sp.b << 16);
          sp_cls[i] = nsh(sp.la) | (nsh(sp.lb) << 8);
          sp_rel[i] = rel;
          fit += rel + nsh(sp.la) * nsh(sp.lb) <= kBlkStage;
          if (i == 0) chunk_base = b0;
        }
      }
      const int cnt = max(1, __syncthreads_count(fit > 0 && tid < nq) +
                                 __syncthreads_count(fit > 1));
      const int last = cnt - 1;
      const int len = sp_rel[last] + (sp_cls[last] & 0xff) * (sp_cls[last] >> 8);
      const double *src = bt + chunk_base;
      for (int t = 0; t < tn; ++t)
        for (int i = tid; i < len; i += kContractThreads)
          cp_async8(&bs[t][i], src + (long long)t * w.blk_total + i);
      asm volatile("cp.async.commit_group;\n" ::: "memory");
      asm volatile("cp.async.wait_group 0;\n" ::: "memory");
      __syncthreads();
      for (int q = 0; q < cnt; ++q) {
        const int ab = sp_ab[q], cl = sp_cls[q];
        const int a = ab & 0xffff, b = ab >> 16, na = cl & 0xff, nb = cl >> 8;
        const int rel = sp_rel[q];
#pragma unroll
        for (int j = 0; j < kElemsPerThread; ++j) {
          if (lm1[j] >= na || lm2[j] >= nb) continue;
          const double cw = cf1[a * ni + m1[j]] * cf2[b * nj + m2[j]];
          const int o = rel + lm1[j] * nb + lm2[j];
#pragma unroll
          for (int t = 0; t < kTermsPerCta; ++t)
            if (t < tn) acc[j][t] += cw * bs[t][o];
        }
      }
      q0 += cnt;
    }
#pragma unroll
    for (int j = 0; j < kElemsPerThread; ++j) {
      const int e = e0 + tid + j * kContractThreads;
      if (e >= ne) continue;
#pragma unroll
      for (int t = 0; t < kTermsPerCta; ++t)
        if (t < tn) M[(long long)(t0 + t) * w.m_total + base + e] = acc[j][t];
    }
  }
}

int launch_contract(const DevSys &s, const DevWork &w, int nterm,
                    const double *blk, double *M, cudaStream_t st, int terms_per_cta) {
  if (w.nunits == 0 || nterm == 0) return IMAGO_OK;
  if (terms_per_cta >= 8 && nterm > 4) {
    const long long grid = (long long)w.nunits * ((nterm + 7) / 8);
    k_contract<8><<<(unsigned)grid, kContractThreads, 0, st>>>(s, w, nterm, blk, M);
  } else {
    const long long grid = (long long)w.nunits * ((nterm + 3) / 4);
    k_contract<4><<<(unsigned)grid, kContractThreads, 0, st>>>(s, w, nterm, blk, M);
  }
  IMAGO_CUDA(cudaGetLastError());
  return IMAGO_OK;
}

// ------------------------------------------------------------- bloch --
// For each atom pair, P(k) = exp(i k.L0) sum_{images u} exp(i k.R_u) M_u:
// a GEMM of the complex phase table [k x u] with the real image blocks
// [u x e], per term.  The result is scattered as saveCurrentPair does
// (valence first, core after, dagger for the transposed core blocks, the
// last write winning for i == j), intgSaving.F90:132-702.
constexpr int kBK = 32;   // k-points per CTA
constexpr int kBC = kBlochCols;  // block elements per CTA
constexpr int kBU = 16;   // images per shared-memory stage

__device__ __forceinline__ void scatter(const DevSys &s, const DPair &p,
                                        long long tk, int m1, int m2,
                                        double re, double im, double2 *vv,
                                        double2 *cv, double2 *cc) {
  const int V = s.vale_dim, C = s.core_dim;
  const int v1 = s.type_nvale[p.ti], v2 = s.type_nvale[p.tj];
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

// ------------------------------------------------------------ K-overlap --
// saveCurrentPair with saveFull = 1 (intgSaving.F90:346-459, 513-551,
// 555-608, 654-690): block (i, j) takes the pair's element, block (j, i)
// its conjugate at the transposed place; for i == j the dagger, written
// second in the reference, replaces the block, so only it is written.
__device__ __forceinline__ void scatter_full(const DevSys &s, const DPair &p,
                                             long long tk, int m1, int m2,
                                             double re, double im, double2 *vv,
                                             double2 *cv, double2 *cc) {
  const int V = s.vale_dim, C = s.core_dim;
  const int v1 = s.type_nvale[p.ti], v2 = s.type_nvale[p.tj];
  const bool same = p.i == p.j;
  if (m1 < v1 && m2 < v2) {
    const int r = s.site_cum_vale[p.i] + m1, c = s.site_cum_vale[p.j] + m2;
    if (!same) vv[tk * V * V + (long long)c * V + r] = make_double2(re, im);
    vv[tk * V * V + (long long)r * V + c] = make_double2(re, -im);
    return;
  }
  if (C == 0) return;
  if (m1 >= v1 && m2 < v2) {
    if (same) return;
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
    if (!same) cc[tk * C * C + (long long)r2 * C + r1] = make_double2(re, im);
    cc[tk * C * C + (long long)r1 * C + r2] = make_double2(re, -im);
  }
}

// Tensor-core phase sum over a (pair, BC-column tile, 32 k-points, term):
// 2 x BC/16 warps, each a 16 k x 16 column tile.  Rows of m_s are BC + 4
// doubles and rows of ph_s 34 complex values, both 8 mod 32 bank words, so
// the 4 k rows of a fragment read fall on distinct banks in each wavefront.
constexpr int kBKP = kBK + 2;

// KOV: the plane-wave overlap's complex blocks, the real and imaginary
// parts being terms 2 z and 2 z + 1 of M (z = blockIdx.z, the wave
// vector): the image loop runs once per part into its own accumulators,
// and the epilogue saves both orientations (scatter_full).
template <int BC, bool KOV = false>
__global__ void __launch_bounds__(4 * BC, (KOV ? 128 : 256) / BC)
    k_bloch(DevSys s, DevWork w, const double *M, double2 *vv, double2 *cv,
            double2 *cc) {
  constexpr int T = 4 * BC, NWC = BC / 16;
  constexpr int PH = (kBU * kBK + T - 1) / T, ML = kBU * BC / T;
  // two stages: the next 16 images load (cp.async) during this stage's MMAs;
  // the epilogue reuses the same shared memory for the output tile
  constexpr size_t kPhBytes = 2 * kBU * kBKP * sizeof(double2);
  constexpr size_t kMBytes = 2 * kBU * (BC + 4) * sizeof(double);
  constexpr size_t kOutBytes = kBK * (BC + 1) * sizeof(double2);
  constexpr size_t kSmBytes =
      kPhBytes + kMBytes > kOutBytes ? kPhBytes + kMBytes : kOutBytes;
  __shared__ __align__(16) unsigned char bsm[kSmBytes];
  auto ph_s = reinterpret_cast<double2(*)[kBU][kBKP]>(bsm);
  auto m_s = reinterpret_cast<double(*)[kBU][BC + 4]>(bsm + kPhBytes);
  const int2 bt = w.btile_w[blockIdx.x];
  const DPair p = w.pairs[bt.x];
  const int ne = p.ni * p.nj, c0 = bt.y * BC;
  const int k0 = blockIdx.y * kBK, term = blockIdx.z, nk = s.nk;
  const int nu = p.uend - p.ubeg;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wk = (warp / NWC) * 16, wc = (warp % NWC) * 16;  // warp tile origin
  constexpr int NP = KOV ? 2 : 1;
  const double *Mt = nullptr;
  double ar[NP][2][2][2] = {}, ai[NP][2][2][2] = {};
  auto issue = [&](int u0, int buf) {
#pragma unroll
    for (int q = 0; q < PH; ++q) {
      const int i = tid + q * T, uu = i / kBK, kk = i % kBK;
      if (i < kBU * kBK) {
        const bool in = u0 + uu < nu && k0 + kk < nk;
        const double2 *src =
            in ? s.phase + (long long)w.units[p.ubeg + u0 + uu].cell * nk + k0 + kk
               : s.phase;
        cp_async16(&ph_s[buf][uu][kk], src, in);
      }
    }
#pragma unroll
    for (int q = 0; q < ML; ++q) {
      const int i = tid + q * T, uu = i / BC, cc2 = i % BC;
      const bool in = u0 + uu < nu && c0 + cc2 < ne;
      cp_async8z(&m_s[buf][uu][cc2], in ? Mt + (long long)(u0 + uu) * ne + c0 + cc2 : Mt,
                 in);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
#pragma unroll
  for (int part = 0; part < NP; ++part) {
  Mt = M + (long long)(KOV ? 2 * term + part : term) * w.m_total + p.moff;
  if (nu > 0) issue(0, 0);
  for (int u0 = 0, buf = 0; u0 < nu; u0 += kBU, buf ^= 1) {
    if (u0 + kBU < nu) {
      issue(u0 + kBU, buf ^ 1);
      asm volatile("cp.async.wait_group 1;\n" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    }
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < kBU; ks += 4) {
      const int ku = ks + (lane & 3);
      double b[2];
      double2 a[2];
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        b[t] = m_s[buf][ku][wc + t * 8 + (lane >> 2)];
        a[t] = ph_s[buf][ku][wk + t * 8 + (lane >> 2)];
      }
#pragma unroll
      for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) {
          dmma(ar[part][mt][nt][0], ar[part][mt][nt][1], a[mt].x, b[nt]);
          dmma(ai[part][mt][nt][0], ai[part][mt][nt][1], a[mt].y, b[nt]);
        }
    }
    __syncthreads();  // this stage's buffer is refilled two stages on
  }
  }
  // epilogue: origin shift (kPointLatticeOriginShift, intgSaving.F90:241-292,
  // skipped when |k.L0| < smallThresh) and the scatter.  The plain form
  // stages the 32 k x BC tile through shared memory (the stages' buffers,
  // free after the last barrier) so that consecutive threads store
  // consecutive block elements of one k-point.
  if constexpr (!KOV) {
    auto out_s = reinterpret_cast<double2(*)[BC + 1]>(bsm);
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
      const int kl = wk + mt * 8 + (lane >> 2), k = k0 + kl;
      double sn = 0.0, cs = 1.0;
      if (k < nk) {
        const double *kv = s.kxyz + 3 * k;
        const double dot = kv[0] * p.L0[0] + kv[1] * p.L0[1] + kv[2] * p.L0[2];
        if (fabs(dot) >= kSmallThresh) sincos(dot, &sn, &cs);
      }
#pragma unroll
      for (int nt = 0; nt < 2; ++nt)
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const double re = ar[0][mt][nt][i], im = ai[0][mt][nt][i];
          const double xr = cs * re - sn * im, xi = cs * im + sn * re;
          out_s[kl][wc + nt * 8 + 2 * (lane & 3) + i] =
              s.minus_i ? make_double2(xi, -xr) : make_double2(xr, xi);
        }
    }
    __syncthreads();
    for (int idx = tid; idx < kBK * BC; idx += T) {
      const int kl = idx / BC, el = idx - kl * BC;
      const int k = k0 + kl, e = c0 + el;
      if (k >= nk || e >= ne) continue;
      const int m2 = e / p.ni, m1 = e - m2 * p.ni;
      const double2 v = out_s[kl][el];
      scatter(s, p, (long long)term * nk + k, m1, m2, v.x, v.y, vv, cv, cc);
    }
  } else {
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
      const int k = k0 + wk + mt * 8 + (lane >> 2);
      if (k >= nk) continue;
      const double *kv = s.kxyz + 3 * k;
      const double dot = kv[0] * p.L0[0] + kv[1] * p.L0[1] + kv[2] * p.L0[2];
      double sn = 0.0, cs = 1.0;
      if (fabs(dot) >= kSmallThresh) sincos(dot, &sn, &cs);
      const long long tk = (long long)term * nk + k;
#pragma unroll
      for (int nt = 0; nt < 2; ++nt)
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const int e = c0 + wc + nt * 8 + 2 * (lane & 3) + i;
          if (e >= ne) continue;
          // KOV: (phase) x (Mr + i Mi)
          const double re = KOV ? ar[0][mt][nt][i] - ai[NP - 1][mt][nt][i] : ar[0][mt][nt][i];
          const double im = KOV ? ai[0][mt][nt][i] + ar[NP - 1][mt][nt][i] : ai[0][mt][nt][i];
          const int m2 = e / p.ni, m1 = e - m2 * p.ni;
          const double xr = cs * re - sn * im, xi = cs * im + sn * re;
          if (KOV)
            scatter_full(s, p, tk, m1, m2, xr, xi, vv, cv, cc);
          else if (s.minus_i)
            scatter(s, p, tk, m1, m2, xi, -xr, vv, cv, cc);
          else
            scatter(s, p, tk, m1, m2, xr, xi, vv, cv, cc);
        }
    }
  }
}

// Few k-points (Gamma, 2x2x2): the tensor-core tiles would idle on k, so
// one thread per block column keeps the nk complex sums in registers and
// reads each image block once.

__global__ void __launch_bounds__(kBC)
    k_bloch_small(DevSys s, DevWork w, const double *M, double2 *vv,
                  double2 *cv, double2 *cc) {
  __shared__ double2 shift[kBlochSmallNk];
  const int2 bt = w.btile[blockIdx.x];
  const DPair p = w.pairs[bt.x];
  const int ne = p.ni * p.nj, e = bt.y * kBC + threadIdx.x;
  const int term = blockIdx.y, nk = s.nk;
  if (threadIdx.x < nk) {
    // kPointLatticeOriginShift (intgSaving.F90:241-292)
    const double *kv = s.kxyz + 3 * threadIdx.x;
    const double dot = kv[0] * p.L0[0] + kv[1] * p.L0[1] + kv[2] * p.L0[2];
    double sn = 0.0, cs = 1.0;
    if (fabs(dot) >= kSmallThresh) sincos(dot, &sn, &cs);
    shift[threadIdx.x] = make_double2(cs, sn);
  }
  __syncthreads();
  if (e >= ne) return;
  const double *Mt = M + (long long)term * w.m_total + p.moff + e;
  double re[kBlochSmallNk], im[kBlochSmallNk];
#pragma unroll
  for (int k = 0; k < kBlochSmallNk; ++k) re[k] = im[k] = 0.0;
  for (int u = p.ubeg; u < p.uend; ++u) {
    const double m = Mt[(long long)(u - p.ubeg) * ne];
    const double2 *ph = s.phase + (long long)w.units[u].cell * nk;
#pragma unroll
    for (int k = 0; k < kBlochSmallNk; ++k)
      if (k < nk) {
        const double2 f = ph[k];
        re[k] += f.x * m;
        im[k] += f.y * m;
      }
  }
  const int m2 = e / p.ni, m1 = e - m2 * p.ni;
#pragma unroll
  for (int k = 0; k < kBlochSmallNk; ++k)
    if (k < nk) {
      const double2 f = shift[k];
      const double xr = f.x * re[k] - f.y * im[k], xi = f.x * im[k] + f.y * re[k];
      if (s.minus_i)
        scatter(s, p, (long long)term * nk + k, m1, m2, xi, -xr, vv, cv, cc);
      else
        scatter(s, p, (long long)term * nk + k, m1, m2, xr, xi, vv, cv, cc);
    }
}

int launch_bloch(const DevSys &s, const DevWork &w, int nterm, const double *M,
                 double2 *vv, double2 *cv, double2 *cc, cudaStream_t st) {
  if (w.nbtile == 0 || nterm == 0) return IMAGO_OK;
  if (s.nk <= kBlochSmallNk) {
    k_bloch_small<<<dim3(w.nbtile, nterm), kBC, 0, st>>>(s, w, M, vv, cv, cc);
    IMAGO_CUDA(cudaGetLastError());
    return IMAGO_OK;
  }
  dim3 grid(w.nbtile_w, (s.nk + kBK - 1) / kBK, nterm);
  if (w.nbtile_w == 0) return IMAGO_OK;
  switch (w.bw) {
    case bloch_width(0):
      k_bloch<bloch_width(0)><<<grid, 4 * bloch_width(0), 0, st>>>(s, w, M, vv, cv, cc);
      break;
    case bloch_width(1):
      k_bloch<bloch_width(1)><<<grid, 4 * bloch_width(1), 0, st>>>(s, w, M, vv, cv, cc);
      break;
    case bloch_width(2):
      k_bloch<bloch_width(2)><<<grid, 4 * bloch_width(2), 0, st>>>(s, w, M, vv, cv, cc);
      break;
    default:
      return IMAGO_ERR_INVALID;
  }
  IMAGO_CUDA(cudaGetLastError());
  return IMAGO_OK;
}

// ------------------------------------------------------------- ortho --
// With S = coreValeOL and X the matrix being orthogonalised, the reference
// computes (zherk or zher2k on the upper triangle, then coreValeCoreCore
// and makeValeVale):
//   VV' = VV - S^H X_cv - X_cv^H S + S^H X_cc S.
// Here it is formed as VV' = VV - (S^H Y + Y^H S) with Y = X_cv - X_cc S/2
// (X_cc is Hermitian), two complex GEMMs on 32x32 output tiles:
//   k_ortho_y: Y (C x V),  k_ortho_w: the upper tiles of S^H Y + Y^H S,
// then the packing of the upper triangle with the 1e-10 zeroing.
// For the overlap itself X = S: VV - 2 S^H S + S^H S_cc S.
constexpr int kOT = 32;   // output tile
constexpr int kOK = 16;   // complex K per shared-memory stage
constexpr int kOP = kOT + 2;  // 34 double2 = 136 bank words: conflict-free fragment reads
constexpr int kOThreads = 128;
constexpr int kOLoads = kOK * kOT / kOThreads;  // double2 per thread per operand

// Shared operands of one stage: A(k, r) and B(k, c), complex, interleaved.
struct OStage {
  double2 a[kOK][kOP];
  double2 b[kOK][kOP];
};

// Accumulate the stage into the warp's 16x16 complex tile, op(A)^T B with
// op = conj when CONJ, by three real products per complex one (the 3M
// form): t1 += ar br, t2 += ai bi, t3 += (ar -/+ ai)(br + bi).  Then
//   CONJ:  re = t1 + t2, im = t3 - t1 + t2
//   plain: re = t1 - t2, im = t3 - t1 - t2.
// Warp w owns rows 16*(w/2).. and columns 16*(w%2)..
template <bool CONJ, bool REAL>
__device__ __forceinline__ void ostage_mma(const OStage &st, double t1[2][2][2],
                                           double t2[2][2][2], double t3[2][2][2],
                                           int lane, int warp) {
  const int r0 = (warp >> 1) * 16, cb = (warp & 1) * 16;
#pragma unroll
  for (int ks = 0; ks < kOK; ks += 4) {
    const int kk = ks + (lane & 3);
    double2 a[2], b[2];
    double as[2], bs[2];
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      a[t] = st.a[kk][r0 + 8 * t + (lane >> 2)];
      b[t] = st.b[kk][cb + 8 * t + (lane >> 2)];
      as[t] = CONJ ? a[t].x - a[t].y : a[t].x + a[t].y;
      bs[t] = b[t].x + b[t].y;
    }
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
      for (int nt = 0; nt < 2; ++nt) {
        dmma(t1[mt][nt][0], t1[mt][nt][1], a[mt].x, b[nt].x);
        if (REAL) continue;  // imaginary parts are zero: t2 = 0, t3 = t1
        dmma(t2[mt][nt][0], t2[mt][nt][1], a[mt].y, b[nt].y);
        dmma(t3[mt][nt][0], t3[mt][nt][1], as[mt], bs[nt]);
      }
  }
}

// Complex tile entry from the three 3M sums.
template <bool CONJ, bool REAL>
__device__ __forceinline__ double2 ocombine(double t1, double t2, double t3) {
  if (REAL) return make_double2(t1, 0.0);
  return CONJ ? make_double2(t1 + t2, t3 - t1 + t2)
              : make_double2(t1 - t2, t3 - t1 - t2);
}

// Y(c, v) = X_cv(c, v) - ycc sum_l X_cc(c, l) S(l, v), ycc = 1/2 for a
// Hermitian X_cc (the her2k form) and 1 for the general form below.
// Operands are staged through registers one K stage ahead of the MMAs.
template <bool REAL>
__global__ void __launch_bounds__(kOThreads, 4)
    k_ortho_y(DevSys s, const double2 *cv, const double2 *cc,
              const double2 *s_cv, double2 *y, double ycc) {
  __shared__ OStage st;
  const int V = s.vale_dim, C = s.core_dim;
  const int ntc = (C + kOT - 1) / kOT;
  const int tr = blockIdx.x % ntc, tc = blockIdx.x / ntc;  // c tile, v tile
  const int k = blockIdx.y, term = blockIdx.z;
  const long long tk = (long long)term * s.nk + k;
  const double2 *XC = cc + tk * C * C;
  const double2 *S = s_cv + (long long)k * V * C;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double t1[2][2][2] = {}, t2[2][2][2] = {}, t3[2][2][2] = {};
  double2 ra[kOLoads], rb[kOLoads];
  auto fetch = [&](int l0) {
#pragma unroll
    for (int q = 0; q < kOLoads; ++q) {
      const int i = tid + q * kOThreads;
      // A: X_cc(c, l), c fastest in memory
      const int ar = i % kOT, ak = i / kOT;
      const int l = l0 + ak, c = tr * kOT + ar;
      ra[q] = (l < C && c < C) ? XC[(long long)l * C + c] : make_double2(0.0, 0.0);
      // B: S(l, v), l fastest in memory
      const int bk = i % kOK, br = i / kOK;
      const int lb = l0 + bk, v = tc * kOT + br;
      rb[q] = (lb < C && v < V) ? S[(long long)v * C + lb] : make_double2(0.0, 0.0);
    }
  };
  auto store = [&]() {
#pragma unroll
    for (int q = 0; q < kOLoads; ++q) {
      const int i = tid + q * kOThreads;
      st.a[i / kOT][i % kOT] = ra[q];
      st.b[i % kOK][i / kOK] = rb[q];
    }
  };
  fetch(0);
  for (int l0 = 0; l0 < C; l0 += kOK) {
    __syncthreads();
    store();
    __syncthreads();
    if (l0 + kOK < C) fetch(l0 + kOK);
    ostage_mma<false, REAL>(st, t1, t2, t3, lane, warp);
  }
  const double2 *X = cv + tk * V * C;
  double2 *Y = y + tk * V * C;
  const int r0 = (warp >> 1) * 16, cb = (warp & 1) * 16;
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < 2; ++nt)
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int c = tr * kOT + r0 + 8 * mt + (lane >> 2);
        const int v = tc * kOT + cb + 8 * nt + 2 * (lane & 3) + i;
        if (c >= C || v >= V) continue;
        const double2 x = X[(long long)v * C + c];
        const double2 p = ocombine<false, REAL>(t1[mt][nt][i], t2[mt][nt][i], t3[mt][nt][i]);
        Y[(long long)v * C + c] = make_double2(x.x - ycc * p.x, x.y - ycc * p.y);
      }
}

// Upper tiles (J <= I) of W = S^H Y + X2^H S as one K loop over the stacked
// core index (S;X2)^H (Y;S), then VV'(j, i) = VV(j, i) - W(j, i) packed at
// i(i+1)/2 + j.  The her2k form passes X2 = Y and makes the diagonal real;
// the general form (`general`, X2 = X_cv, Y = X_cv - X_cc S) keeps on the
// diagonal the imaginary part of S^H X_cc S = -Im W there.
template <bool REAL, bool FULL = false>
__global__ void __launch_bounds__(kOThreads, 4)
    k_ortho_w(DevSys s, const double2 *vv, const double2 *y, const double2 *x2,
              const double2 *s_cv, double *packed, bool general, double *im_plane = nullptr) {
  __shared__ OStage st;
  const int V = s.vale_dim, C = s.core_dim;
  // upper-triangular tile index -> (J, I), J <= I; FULL: every tile
  int I = 0, J = 0;
  if (FULL) {
    const int tvv = (V + kOT - 1) / kOT;
    J = blockIdx.x % tvv;
    I = blockIdx.x / tvv;
  } else {
    int t = blockIdx.x;
    while (t > I) {
      t -= I + 1;
      ++I;
    }
    J = t;
  }
  const int k = blockIdx.y, term = blockIdx.z;
  const long long tk = (long long)term * s.nk + k;
  const double2 *S = s_cv + (long long)k * V * C;
  const double2 *Y = y + tk * V * C, *X2 = x2 + tk * V * C;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int K2 = 2 * C;
  double t1[2][2][2] = {}, t2[2][2][2] = {}, t3[2][2][2] = {};
  // on a diagonal tile the warp owning rows 16..31 x columns 0..15 lies
  // wholly below the diagonal, which is never stored
  const bool lower = !FULL && J == I && (warp >> 1) > (warp & 1);
  double2 ra[kOLoads], rb[kOLoads];
  auto fetch = [&](int l0) {
#pragma unroll
    for (int q = 0; q < kOLoads; ++q) {
      const int i = tid + q * kOThreads;
      const int kk = i % kOK, r = i / kOK;
      const int l = l0 + kk;
      const int j = J * kOT + r, ii = I * kOT + r;
      double2 a = make_double2(0.0, 0.0), b = make_double2(0.0, 0.0);
      if (l < K2) {
        const double2 *Aop = l < C ? S : X2;  // (S; X2), conjugated in the MMA
        const double2 *Bop = l < C ? Y : S;   // (Y; S)
        const int lc = l < C ? l : l - C;
        if (j < V) a = Aop[(long long)j * C + lc];
        if (ii < V) b = Bop[(long long)ii * C + lc];
      }
      ra[q] = a;
      rb[q] = b;
    }
  };
  auto store = [&]() {
#pragma unroll
    for (int q = 0; q < kOLoads; ++q) {
      const int i = tid + q * kOThreads;
      st.a[i % kOK][i / kOK] = ra[q];
      st.b[i % kOK][i / kOK] = rb[q];
    }
  };
  fetch(0);
  for (int l0 = 0; l0 < K2; l0 += kOK) {
    __syncthreads();
    store();
    __syncthreads();
    if (l0 + kOK < K2) fetch(l0 + kOK);
    if (!lower) ostage_mma<true, REAL>(st, t1, t2, t3, lane, warp);
  }
  const double2 *VVt = vv + tk * V * V;
  const long long np = (long long)V * (V + 1) / 2;
  double *out = packed + 2 * tk * np;
  const int r0 = (warp >> 1) * 16, cb = (warp & 1) * 16;
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < 2; ++nt)
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int row = J * kOT + r0 + 8 * mt + (lane >> 2);
        const int col = I * kOT + cb + 8 * nt + 2 * (lane & 3) + i;
        if (row >= V || col >= V || (!FULL && row > col)) continue;
        double2 v = VVt[(long long)col * V + row];
        const double2 p = ocombine<true, REAL>(t1[mt][nt][i], t2[mt][nt][i], t3[mt][nt][i]);
        v.x -= p.x;
        v.y -= p.y;
        if (FULL) {  // the whole matrix as real and imaginary planes
          const long long o = (tk * V + col) * (long long)V + row;
          packed[o] = v.x;
          im_plane[o] = v.y;
          continue;
        }
        if (row == col) v.y = general ? -p.y : 0.0;  // zher2k keeps it real
        if (fabs(v.x) < kPackThresh) v.x = 0.0;
        if (fabs(v.y) < kPackThresh) v.y = 0.0;
        const long long idx = (long long)col * (col + 1) / 2 + row;
        store_packed(out, idx, v);
      }
}

// Small systems: the whole orthogonalisation of one (k, term) in one CTA.
// S (C x V), X_cv (C x V) and X_cc (C x C) are read once into shared
// memory (k-major rows, zero padded to multiples of 4 in k and 16 in the
// output index, rows of 2 mod 8 complex values for conflict-free fragment
// reads); Y = X_cv - X_cc S / 2 is formed in place of X_cv, then the upper
// 16x16 subtiles of S^H Y + Y^H S are taken straight from shared memory and
// subtracted from VV in the packing epilogue.  Used while the three arrays
// fit in kFusedMaxSmem.
constexpr int kFThreads = 512;
constexpr int kFWarps = kFThreads / 32;
constexpr size_t kFusedMaxSmem = 200 * 1024;

struct FusedDims {
  int C4, C16, V16, Vp, Cp;
};

__host__ __device__ inline FusedDims fused_dims(int C, int V) {
  FusedDims d;
  d.C4 = (C + 3) / 4 * 4;
  d.C16 = (C + 15) / 16 * 16;
  d.V16 = (V + 15) / 16 * 16;
  d.Vp = d.V16 + 2;
  d.Cp = d.C16 + 2;
  return d;
}

inline size_t fused_smem(int C, int V) {
  const FusedDims d = fused_dims(C, V);
  return sizeof(double2) * ((size_t)2 * d.C4 * d.Vp + (size_t)d.C4 * d.Cp);
}

// One warp's 16x16 complex subtile of op(A)^T B over k in [k0, k0 + nk4)
// from k-major shared arrays (row strides lda, ldb), 3M form.
template <bool CONJ, bool REAL>
__device__ __forceinline__ void fused_tile(const double2 *A, int lda, int r0,
                                           const double2 *B, int ldb, int c0,
                                           int nk4, bool skip_lower,
                                           double t1[2][2][2], double t2[2][2][2],
                                           double t3[2][2][2], int lane) {
  for (int ks = 0; ks < nk4; ks += 4) {
    const int kk = ks + (lane & 3);
    double2 a[2], b[2];
    double as[2], bs[2];
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      a[t] = A[kk * lda + r0 + 8 * t + (lane >> 2)];
      b[t] = B[kk * ldb + c0 + 8 * t + (lane >> 2)];
      as[t] = CONJ ? a[t].x - a[t].y : a[t].x + a[t].y;
      bs[t] = b[t].x + b[t].y;
    }
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
      for (int nt = 0; nt < 2; ++nt) {
        if (skip_lower && mt > nt) continue;  // rows 8..15 x cols 0..7
        dmma(t1[mt][nt][0], t1[mt][nt][1], a[mt].x, b[nt].x);
        if (REAL) continue;  // imaginary parts are zero: t2 = 0, t3 = t1
        dmma(t2[mt][nt][0], t2[mt][nt][1], a[mt].y, b[nt].y);
        dmma(t3[mt][nt][0], t3[mt][nt][1], as[mt], bs[nt]);
      }
  }
}

// One warp's 8x16 complex subtile of A^T B (plain, 3M form) over k in
// [0, nk4) from k-major shared arrays: one row fragment, two column ones.
template <bool REAL>
__device__ __forceinline__ void fused_tile8(const double2 *A, int lda, int r0,
                                            const double2 *B, int ldb, int c0, int nk4,
                                            double t1[2][2], double t2[2][2],
                                            double t3[2][2], int lane) {
  for (int ks = 0; ks < nk4; ks += 4) {
    const int kk = ks + (lane & 3);
    const double2 a = A[kk * lda + r0 + (lane >> 2)];
    const double as = a.x + a.y;
    double2 b[2];
    double bs[2];
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      b[t] = B[kk * ldb + c0 + 8 * t + (lane >> 2)];
      bs[t] = b[t].x + b[t].y;
    }
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) {
      dmma(t1[nt][0], t1[nt][1], a.x, b[nt].x);
      if (REAL) continue;
      dmma(t2[nt][0], t2[nt][1], a.y, b[nt].y);
      dmma(t3[nt][0], t3[nt][1], as, bs[nt]);
    }
  }
}

// Y tiles of 8 core x 16 valence indices held per warp before X_cv lands
constexpr int kFYTilesPerWarp = 3;

template <bool REAL>
__global__ void __launch_bounds__(kFThreads, 1)
    k_ortho_fused(DevSys s, const double2 *vv, const double2 *cv,
                  const double2 *cc, const double2 *s_cv, double *packed) {
  extern __shared__ double2 fsm[];
  const int V = s.vale_dim, C = s.core_dim;
  const FusedDims d = fused_dims(C, V);
  double2 *Ss = fsm, *Ys = fsm + d.C4 * d.Vp, *Xs = Ys + d.C4 * d.Vp;
  const int k = blockIdx.x, term = blockIdx.y;
  const long long tk = (long long)term * s.nk + k;
  const double2 *S = s_cv + (long long)k * V * C;
  const double2 *X = cv + tk * V * C;
  const double2 *XC = cc + tk * C * C;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // S(l, v) and X_cc(c, l) first (S to [l][v], X_cc to [l][c], l and c
  // fastest in memory), then X_cv(l, v) to [l][v] in a second group that
  // lands while the products of the Y step run: asynchronous 16-byte
  // copies, the padding zero-filled
  for (int i = tid; i < d.C4 * d.V16; i += kFThreads) {
    const int l = i % d.C4, v = i / d.C4;
    const bool in = l < C && v < V;
    cp_async16(&Ss[l * d.Vp + v], S + (in ? (long long)v * C + l : 0), in);
  }
  for (int i = tid; i < d.C4 * d.C16; i += kFThreads) {
    const int c = i % d.C16, l = i / d.C16;
    const bool in = l < C && c < C;
    cp_async16(&Xs[l * d.Cp + c], XC + (in ? (long long)l * C + c : 0), in);
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  for (int i = tid; i < d.C4 * d.V16; i += kFThreads) {
    const int l = i % d.C4, v = i / d.C4;
    const bool in = l < C && v < V;
    cp_async16(&Ys[l * d.Vp + v], X + (in ? (long long)v * C + l : 0), in);
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  asm volatile("cp.async.wait_group 1;\n" ::: "memory");
  __syncthreads();
  // Y = X_cv - X_cc S / 2 on tiles of 8 core x 16 valence indices (C = 40
  // gives 5 row tiles, no padding): each warp forms the products of its
  // tiles (at most kFYTilesPerWarp) in registers, then, once X_cv is in,
  // subtracts them
  const int yr = (C + 7) / 8, ny = yr * (d.V16 / 16);
  double y1[kFYTilesPerWarp][2][2], y2[kFYTilesPerWarp][2][2], y3[kFYTilesPerWarp][2][2];
#pragma unroll
  for (int q = 0; q < kFYTilesPerWarp; ++q) {
    const int tile = warp + q * kFWarps;
#pragma unroll
    for (int nt = 0; nt < 2; ++nt)
#pragma unroll
      for (int i = 0; i < 2; ++i) y1[q][nt][i] = y2[q][nt][i] = y3[q][nt][i] = 0.0;
    if (tile < ny)
      fused_tile8<REAL>(Xs, d.Cp, (tile % yr) * 8, Ss, d.Vp, (tile / yr) * 16, d.C4, y1[q],
                        y2[q], y3[q], lane);
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  __syncthreads();
#pragma unroll
  for (int q = 0; q < kFYTilesPerWarp; ++q) {
    const int tile = warp + q * kFWarps;
    if (tile >= ny) continue;
    const int r0 = (tile % yr) * 8, c0 = (tile / yr) * 16;
#pragma unroll
    for (int nt = 0; nt < 2; ++nt)
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int c = r0 + (lane >> 2);
        const int v = c0 + 8 * nt + 2 * (lane & 3) + i;
        if (c >= C || v >= V) continue;
        const double2 p = ocombine<false, REAL>(y1[q][nt][i], y2[q][nt][i], y3[q][nt][i]);
        double2 &y = Ys[c * d.Vp + v];
        y.x -= 0.5 * p.x;
        y.y -= 0.5 * p.y;
      }
  }
  __syncthreads();
  // upper subtiles (J <= I) of S^H Y + Y^H S over the stacked k = 2 C4
  const double2 *VVt = vv + tk * V * V;
  const long long np = (long long)V * (V + 1) / 2;
  double *out = packed + 2 * tk * np;
  const int nt16 = d.V16 / 16, nup = nt16 * (nt16 + 1) / 2;
  for (int tile = warp; tile < nup; tile += kFWarps) {
    int t = tile, I = 0;
    while (t > I) {
      t -= I + 1;
      ++I;
    }
    const int J = t, r0 = J * 16, c0 = I * 16;
    // the tile's VV entries, loaded before the MMAs so they arrive meanwhile
    double2 vvp[2][2][2];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
      for (int nt = 0; nt < 2; ++nt)
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const int row = r0 + 8 * mt + (lane >> 2);
          const int col = c0 + 8 * nt + 2 * (lane & 3) + i;
          vvp[mt][nt][i] = (row < V && col < V && row <= col)
                               ? VVt[(long long)col * V + row]
                               : make_double2(0.0, 0.0);
        }
    double t1[2][2][2] = {}, t2[2][2][2] = {}, t3[2][2][2] = {};
    fused_tile<true, REAL>(Ss, d.Vp, r0, Ys, d.Vp, c0, d.C4, J == I, t1, t2, t3, lane);
    fused_tile<true, REAL>(Ys, d.Vp, r0, Ss, d.Vp, c0, d.C4, J == I, t1, t2, t3, lane);
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
      for (int nt = 0; nt < 2; ++nt)
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const int row = r0 + 8 * mt + (lane >> 2);
          const int col = c0 + 8 * nt + 2 * (lane & 3) + i;
          if (row >= V || col >= V || row > col) continue;
          double2 v = vvp[mt][nt][i];
          const double2 p = ocombine<true, REAL>(t1[mt][nt][i], t2[mt][nt][i], t3[mt][nt][i]);
          v.x -= p.x;
          v.y -= p.y;
          if (row == col) v.y = 0.0;  // zherk/zher2k keep the diagonal real
          if (fabs(v.x) < kPackThresh) v.x = 0.0;
          if (fabs(v.y) < kPackThresh) v.y = 0.0;
          const long long idx = (long long)col * (col + 1) / 2 + row;
          store_packed(out, idx, v);
        }
  }
}

// ----------------------------------------------------- ortho, piped --
// The fused orthogonalisation for builds of several terms as a persistent
// kernel: one CTA per SM walks a contiguous range of (k, term) items in
// k-major order.  S(k) stays in shared memory while k is unchanged; X_cv
// and X_cc of the next item come in by TMA tensor copies (completing on an
// mbarrier) into the second of two X_cv buffers and the X_cc buffer while
// the current item's products run, so the fills hide behind the
// tensor-core work.  S and X_cv are stored in groups of four core indices:
// element (v, k) at ((k / 4) V + v) 4 + k % 4, one 64-byte TMA box row per
// (v, group), which puts the two rows and four k of a quarter warp's
// fragment read on eight distinct 16-byte bank groups without padding;
// X_cc keeps the global layout (core index c fastest) in rows of ld = 2 mod
// 8 complex values, conflict-free for the same reads.  Rows v >= V are not
// stored; their fragments read zero.
struct PipeDims {
  int C4, C16, V16, ld, nbox;
  size_t buf;   // bytes of one S or X_cv array (V x C4 complex), 1024-aligned
  size_t xbuf;  // bytes of the X_cc array (C4 rows of ld complex)
};

__host__ __device__ inline PipeDims pipe_dims(int C, int V) {
  PipeDims d;
  d.C4 = (C + 3) / 4 * 4;
  d.C16 = (C + 15) / 16 * 16;
  d.V16 = (V + 15) / 16 * 16;
  d.nbox = d.C4 / 4;
  d.ld = d.C4 + ((2 - d.C4 % 8) + 8) % 8;
  d.buf = ((size_t)V * d.C4 * sizeof(double2) + 1023) / 1024 * 1024;
  d.xbuf = ((size_t)d.C4 * d.ld * sizeof(double2) + 127) / 128 * 128;
  return d;
}

// dynamic shared memory of k_ortho_pipe at most: 227 KB less room for its
// static shared state
constexpr size_t kPipeMaxSmem = 227 * 1024 - 1024;

inline size_t pipe_smem(int C, int V) {
  const PipeDims d = pipe_dims(C, V);
  return 3 * d.buf + d.xbuf + 64;
}

bool ortho_pipe_fits(int C, int V) {
  const PipeDims d = pipe_dims(C, V);
  return C > 0 && V > 0 && V <= 256 && d.C4 <= 256 && 2 * d.ld <= 256 &&
         pipe_smem(C, V) <= kPipeMaxSmem;
}

// Element (v, k) of an S or X_cv array in groups of four k.
__device__ __forceinline__ int pv(int V, int v, int k) { return (((k >> 2) * V + v) << 2) + (k & 3); }

// One warp's 16x16 complex subtile of op(A)^T B over k in [0, nk4), A and B
// grouped arrays (rows v); rows at or beyond V read as zero.  3M form as
// fused_tile.
template <bool CONJ, bool REAL>
__device__ __forceinline__ void pipe_tile(const double2 *A, int r0, const double2 *B, int c0,
                                          int V, int nk4, bool skip_lower, double t1[2][2][2],
                                          double t2[2][2][2], double t3[2][2][2], int lane) {
  const int ra0 = r0 + (lane >> 2), cb0 = c0 + (lane >> 2);
  const bool va[2] = {ra0 < V, ra0 + 8 < V}, vb[2] = {cb0 < V, cb0 + 8 < V};
  for (int ks = 0; ks < nk4; ks += 4) {
    const int kk = ks + (lane & 3);
    double2 a[2], b[2];
    double as[2], bs[2];
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      a[t] = va[t] ? A[pv(V, ra0 + 8 * t, kk)] : make_double2(0.0, 0.0);
      b[t] = vb[t] ? B[pv(V, cb0 + 8 * t, kk)] : make_double2(0.0, 0.0);
      as[t] = CONJ ? a[t].x - a[t].y : a[t].x + a[t].y;
      bs[t] = b[t].x + b[t].y;
    }
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
      for (int nt = 0; nt < 2; ++nt) {
        if (skip_lower && mt > nt) continue;
        dmma(t1[mt][nt][0], t1[mt][nt][1], a[mt].x, b[nt].x);
        if (REAL) continue;
        dmma(t2[mt][nt][0], t2[mt][nt][1], a[mt].y, b[nt].y);
        dmma(t3[mt][nt][0], t3[mt][nt][1], as[mt], bs[nt]);
      }
  }
}

// The Y step's product X_cc S on an 8 core x 16 valence tile: A(l, c) =
// X_cc(c, l) from the shared [l][c] array (row pitch ld), B(l, v) = S(l, v)
// from the grouped array.
template <bool REAL>
__device__ __forceinline__ void pipe_y_tile(const double2 *XC, int ld, int C, int r0,
                                            const double2 *S, int V, int c0, int nk4,
                                            double t1[2][2], double t2[2][2], double t3[2][2],
                                            int lane) {
  const int ra = r0 + (lane >> 2), cb0 = c0 + (lane >> 2);
  const bool va = ra < C, vb[2] = {cb0 < V, cb0 + 8 < V};
  for (int ks = 0; ks < nk4; ks += 4) {
    const int kk = ks + (lane & 3);
    const double2 a = va ? XC[kk * ld + ra] : make_double2(0.0, 0.0);
    const double as = a.x + a.y;
    double2 b[2];
    double bs[2];
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      b[t] = vb[t] ? S[pv(V, cb0 + 8 * t, kk)] : make_double2(0.0, 0.0);
      bs[t] = b[t].x + b[t].y;
    }
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) {
      dmma(t1[nt][0], t1[nt][1], a.x, b[nt].x);
      if (REAL) continue;
      dmma(t2[nt][0], t2[nt][1], a.y, b[nt].y);
      dmma(t3[nt][0], t3[nt][1], as, bs[nt]);
    }
  }
}

// What every thread of a k_ortho_pipe CTA reads (kept in shared memory,
// written once by thread 0).
struct PipeCta {
  const double2 *vv;
  double *packed;
  double2 *Ss, *Xb[2], *Xc;
  uint64_t *bar;       // S, X buffer 0, X buffer 1
  int *ctr;            // task counters, one per phase parity
  int V, C, nk, nterm, ld, C4, nbox, nup, ny, yr;
  unsigned tx_s, tx_x; // bytes of the S copy; of one item's X_cv and X_cc copies
  long long np, i0;
};

// One W tile (J <= I, the upper 16x16 subtiles of S^H Y + Y^H S) of item q:
// subtracted from VV and packed.
template <bool REAL>
__device__ __forceinline__ void pipe_w_task(const PipeCta &p, long long q, int tile, int lane) {
  const int V = p.V;
  const long long tk = (long long)(q % p.nterm) * p.nk + q / p.nterm;
  const double2 *Ys = p.Xb[(q - p.i0) & 1];
  const double2 *VVt = p.vv + tk * V * V;
  double *out = p.packed + 2 * tk * p.np;
  int t = tile, I = 0;
  while (t > I) {
    t -= I + 1;
    ++I;
  }
  const int J = t, r0 = J * 16, c0 = I * 16;
  // VV is read in the epilogue: other warps' products cover its latency
  double t1[2][2][2] = {}, t2[2][2][2] = {}, t3[2][2][2] = {};
  pipe_tile<true, REAL>(p.Ss, r0, Ys, c0, V, p.C4, J == I, t1, t2, t3, lane);
  pipe_tile<true, REAL>(Ys, r0, p.Ss, c0, V, p.C4, J == I, t1, t2, t3, lane);
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < 2; ++nt)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int row = r0 + 8 * mt + (lane >> 2);
        const int col = c0 + 8 * nt + 2 * (lane & 3) + e;
        if (row >= V || col >= V || row > col) continue;
        double2 v = VVt[(long long)col * V + row];
        const double2 d = ocombine<true, REAL>(t1[mt][nt][e], t2[mt][nt][e], t3[mt][nt][e]);
        v.x -= d.x;
        v.y -= d.y;
        if (row == col) v.y = 0.0;
        if (fabs(v.x) < kPackThresh) v.x = 0.0;
        if (fabs(v.y) < kPackThresh) v.y = 0.0;
        store_packed(out, (long long)col * (col + 1) / 2 + row, v);
      }
}

// One Y tile (8 core x 16 valence) of item q: Y = X_cv - X_cc S / 2 in
// place, X_cc from the shared copy of the item.
template <bool REAL>
__device__ __forceinline__ void pipe_y_task(const PipeCta &p, long long q, int tile, int lane) {
  const int C = p.C, V = p.V;
  double2 *Ys = p.Xb[(q - p.i0) & 1];
  const int r0 = (tile % p.yr) * 8, c0 = (tile / p.yr) * 16;
  double t1[2][2] = {}, t2[2][2] = {}, t3[2][2] = {};
  pipe_y_tile<REAL>(p.Xc, p.ld, C, r0, p.Ss, V, c0, p.C4, t1, t2, t3, lane);
#pragma unroll
  for (int nt = 0; nt < 2; ++nt)
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int c = r0 + (lane >> 2);
      const int v = c0 + 8 * nt + 2 * (lane & 3) + e;
      if (c >= C || v >= V) continue;
      const double2 d = ocombine<false, REAL>(t1[nt][e], t2[nt][e], t3[nt][e]);
      double2 &y = Ys[pv(V, v, c)];
      y.x -= 0.5 * d.x;
      y.y -= 0.5 * d.y;
    }
}

// The copies of item q's X_cv (nbox boxes of four core indices) into buffer
// b and of its X_cc into the X_cc buffer, all completing on bar[1 + b].
__device__ __forceinline__ void pipe_issue_x(const PipeCta &p, long long q, int b,
                                             const CUtensorMap *map_x,
                                             const CUtensorMap *map_c) {
  const int z = (int)((q % p.nterm) * p.nk + q / p.nterm);
  fence_proxy_async();
  mbar_expect_tx(&p.bar[1 + b], p.tx_x);
  for (int g = 0; g < p.nbox; ++g)
    tma_load_3d(p.Xb[b] + (size_t)g * p.V * 4, map_x, &p.bar[1 + b], 8 * g, 0, z);
  tma_load_3d(p.Xc, map_c, &p.bar[1 + b], 0, 0, z);
}

// S(k) into its buffer (nbox boxes), completing on bar[0].
__device__ __forceinline__ void pipe_issue_s(const PipeCta &p, int k, const CUtensorMap *map_s) {
  fence_proxy_async();
  mbar_expect_tx(&p.bar[0], p.tx_s);
  for (int g = 0; g < p.nbox; ++g)
    tma_load_3d(p.Ss + (size_t)g * p.V * 4, map_s, &p.bar[0], 8 * g, 0, k);
}

// One phase between two CTA barriers: the W tiles of item wq (wq < 0: none)
// first, then the Y tiles of item yq (yq < 0: none), handed to warps one
// tile at a time from the phase's counter so that the two kinds balance.
// Y tiles wait (bounded) for their item's copies.  At the start, the
// counter of the next phase is cleared, and the copies of item xq (xq < 0:
// none) are sent for: its X_cv buffer and the X_cc buffer were last read by
// the phase before, which ended at a barrier.  px holds the parity of each
// X barrier's next completion.  False (on every thread) when a copy did not
// land in time.
template <bool REAL>
__device__ __forceinline__ bool pipe_phase(const PipeCta &p, unsigned px[2], int &ph,
                                           long long wq, long long yq, long long xq,
                                           const CUtensorMap *map_x,
                                           const CUtensorMap *map_c) {
  const int tid = threadIdx.x, lane = tid & 31;
  if (tid == 0) {
    p.ctr[ph ^ 1] = 0;
    if (xq >= 0) pipe_issue_x(p, xq, (int)((xq - p.i0) & 1), map_x, map_c);
  }
  const int nw = wq >= 0 ? p.nup : 0, ntask = nw + (yq >= 0 ? p.ny : 0);
  const int yb = yq >= 0 ? (int)((yq - p.i0) & 1) : 0;
  bool ready = false, fail = false;
  while (true) {
    int task = 0;
    if (lane == 0) task = atomicAdd(&p.ctr[ph], 1);
    task = __shfl_sync(0xffffffffu, task, 0);
    if (task >= ntask) break;
    if (task < nw) {
      pipe_w_task<REAL>(p, wq, task, lane);
      continue;
    }
    if (!ready) {
      ready = __all_sync(0xffffffffu, mbar_wait_bounded(&p.bar[1 + yb], px[yb]));
      if (!ready) {
        fail = true;
        break;
      }
    }
    pipe_y_task<REAL>(p, yq, task - nw, lane);
  }
  ph ^= 1;
  const bool bad = __syncthreads_or(fail);
  if (yq >= 0 && !bad) px[yb] ^= 1u;
  return !bad;
}

template <bool REAL>
__global__ void __launch_bounds__(kFThreads, 1)
    k_ortho_pipe(DevSys s, const __grid_constant__ CUtensorMap map_x,
                 const __grid_constant__ CUtensorMap map_c,
                 const __grid_constant__ CUtensorMap map_s, const double2 *vv, int nterm,
                 double *packed) {
  extern __shared__ __align__(1024) unsigned char psm[];
  const int V = s.vale_dim, C = s.core_dim, nk = s.nk;
  const PipeDims d = pipe_dims(C, V);
  const long long N = (long long)nk * nterm;
  const long long i0 = N * blockIdx.x / gridDim.x, i1 = N * (blockIdx.x + 1) / gridDim.x;
  if (i0 >= i1) return;
  __shared__ PipeCta p;
  const int tid = threadIdx.x;
  if (tid == 0) {
    p.vv = vv;
    p.packed = packed;
    p.Ss = reinterpret_cast<double2 *>(psm);
    p.Xb[0] = reinterpret_cast<double2 *>(psm + d.buf);
    p.Xb[1] = reinterpret_cast<double2 *>(psm + 2 * d.buf);
    p.Xc = reinterpret_cast<double2 *>(psm + 3 * d.buf);
    p.bar = reinterpret_cast<uint64_t *>(psm + 3 * d.buf + d.xbuf);
    p.ctr = reinterpret_cast<int *>(p.bar + 3);
    p.V = V;
    p.C = C;
    p.nk = nk;
    p.nterm = nterm;
    p.ld = d.ld;
    p.C4 = d.C4;
    p.nbox = d.nbox;
    const int nt16 = d.V16 / 16;
    p.nup = nt16 * (nt16 + 1) / 2;
    p.yr = (C + 7) / 8;  // Y tiles of 8 core indices
    p.ny = p.yr * nt16;
    p.tx_s = (unsigned)(d.nbox * V * 64);
    p.tx_x = p.tx_s + (unsigned)(d.C4 * d.ld * 16);
    p.np = (long long)V * (V + 1) / 2;
    p.i0 = i0;
    for (int b = 0; b < 3; ++b) mbar_init(&p.bar[b], 1);
    p.ctr[0] = p.ctr[1] = 0;
    mbar_init_fence();
  }
  __syncthreads();
  unsigned ps = 0, px[2] = {0u, 0u};
  int ph = 0;
  int k = (int)(i0 / nterm);
  if (tid == 0) pipe_issue_s(p, k, &map_s);
  // S(k): waited for by every thread; on a timeout the copy in flight gets
  // one more bounded wait before the CTA leaves
  auto load_s_wait = [&]() -> bool {
    const bool ok = mbar_wait_bounded(&p.bar[0], ps);
    ps ^= 1u;
    if (!__syncthreads_or(!ok)) return true;
    if (tid == 0) {
      report_status(s.flag, IMAGO_ERR_TIMEOUT);
      mbar_wait_bounded(&p.bar[0], ps ^ 1u);
    }
    return false;
  };
  bool ok = load_s_wait();
  // item i0: its Y tiles alone
  ok = ok && pipe_phase<REAL>(p, px, ph, -1, i0, i0, &map_x, &map_c);
  for (long long q = i0 + 1; ok && q < i1; ++q) {
    const int kq = (int)(q / nterm);
    if (kq == k) {
      ok = pipe_phase<REAL>(p, px, ph, q - 1, q, q, &map_x, &map_c);
      continue;
    }
    // a new k: the previous item's W tiles, then S(kq), then this item's Y
    ok = pipe_phase<REAL>(p, px, ph, q - 1, -1, q, &map_x, &map_c);
    if (!ok) break;
    k = kq;
    if (tid == 0) pipe_issue_s(p, k, &map_s);
    ok = load_s_wait() && pipe_phase<REAL>(p, px, ph, -1, q, -1, &map_x, &map_c);
  }
  if (ok) ok = pipe_phase<REAL>(p, px, ph, i1 - 1, -1, -1, &map_x, &map_c);
  if (!ok && tid == 0) {
    report_status(s.flag, IMAGO_ERR_TIMEOUT);
    // copies still in flight get one more bounded wait before the CTA leaves
    for (int b = 0; b < 2; ++b) mbar_wait_bounded(&p.bar[1 + b], px[b]);
  }
  __syncthreads();
}

// The bounded wait of k_ortho_pipe on a barrier that nothing completes:
// every thread gives up after limit_ns and the status word records it.
__global__ void k_wait_check(int *flag, unsigned long long limit_ns) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_init_fence();
  }
  __syncthreads();
  const bool ok = mbar_wait_bounded(&bar, 0u, limit_ns);
  if (__syncthreads_or(!ok) && threadIdx.x == 0) report_status(flag, IMAGO_ERR_TIMEOUT);
}

int launch_wait_check(int *flag, double limit_ms, cudaStream_t st) {
  const unsigned long long ns = (unsigned long long)(limit_ms * 1e6);
  k_wait_check<<<1, 128, 0, st>>>(flag, ns);
  IMAGO_CUDA(cudaGetLastError());
  return IMAGO_OK;
}

bool encode_tensor_map_f64_3d(CUtensorMap *map, const void *base, const uint64_t dims[3],
                              const uint64_t strides[2], const uint32_t box[3]) {
  using Encode = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                              const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                              const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                              CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static const Encode fn = []() -> Encode {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    return reinterpret_cast<Encode>(p);
  }();
  if (!fn || ((uintptr_t)base & 15) || (strides[0] & 15) || (strides[1] & 15)) return false;
  const cuuint64_t gd[3] = {dims[0], dims[1], dims[2]};
  const cuuint64_t gs[2] = {strides[0], strides[1]};
  const cuuint32_t bx[3] = {box[0], box[1], box[2]};
  const cuuint32_t es[3] = {1, 1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<void *>(base), gd, gs, bx, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The piped orthogonalisation when it applies (several terms, the arrays in
// shared memory, tensor maps accepted); *launched says whether it ran.
int launch_ortho_pipe(const DevSys &s, int nterm, const double2 *vv, const double2 *cv,
                      const double2 *cc, const double2 *s_cv, double *packed, bool *launched,
                      cudaStream_t st) {
  *launched = false;
  const int V = s.vale_dim, C = s.core_dim;
  if (nterm < 2 || !ortho_pipe_fits(C, V)) return IMAGO_OK;
  const PipeDims d = pipe_dims(C, V);
  CUtensorMap mx, mc, ms;
  // X_cv and S: rows of 2C doubles (v), boxes of 8 doubles (four core
  // indices) x V rows; X_cc: rows of 2C doubles (l), one box of 2 ld
  // doubles x C4 rows.  Beyond C, zero fill.
  const uint64_t dx[3] = {2ull * C, (uint64_t)V, (uint64_t)nterm * s.nk};
  const uint64_t ds[3] = {2ull * C, (uint64_t)V, (uint64_t)s.nk};
  const uint64_t dc[3] = {2ull * C, (uint64_t)C, (uint64_t)nterm * s.nk};
  const uint64_t sv[2] = {16ull * C, 16ull * V * C};
  const uint64_t sc[2] = {16ull * C, 16ull * C * C};
  const uint32_t bv[3] = {8u, (uint32_t)V, 1u};
  const uint32_t bc[3] = {2u * d.ld, (uint32_t)d.C4, 1u};
  if (!encode_tensor_map_f64_3d(&mx, cv, dx, sv, bv) ||
      !encode_tensor_map_f64_3d(&ms, s_cv, ds, sv, bv) ||
      !encode_tensor_map_f64_3d(&mc, cc, dc, sc, bc))
    return IMAGO_OK;
  int dev = 0, nsm = 0;
  IMAGO_CUDA(cudaGetDevice(&dev));
  IMAGO_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  static bool attr_set[2][64] = {};
  const size_t smem = pipe_smem(C, V);
  if (dev >= 0 && dev < 64 && !attr_set[s.real_k][dev]) {
    IMAGO_CUDA(cudaFuncSetAttribute(s.real_k ? k_ortho_pipe<true> : k_ortho_pipe<false>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kPipeMaxSmem));
    attr_set[s.real_k][dev] = true;
  }
  const long long N = (long long)nterm * s.nk;
  const unsigned grid = (unsigned)std::min<long long>(nsm, N);
  if (s.real_k)
    k_ortho_pipe<true><<<grid, kFThreads, smem, st>>>(s, mx, mc, ms, vv, nterm, packed);
  else
    k_ortho_pipe<false><<<grid, kFThreads, smem, st>>>(s, mx, mc, ms, vv, nterm, packed);
  IMAGO_CUDA(cudaGetLastError());
  *launched = true;
  return IMAGO_OK;
}

// coreDim == 0: the reference packs valeVale as it is (integrals.F90:3657-3676).
__global__ void __launch_bounds__(256)
    k_pack_plain(DevSys s, const double2 *vv, double *packed) {
  const int k = blockIdx.y, term = blockIdx.z;
  const int V = s.vale_dim;
  const long long np = (long long)V * (V + 1) / 2;
  const long long tk = (long long)term * s.nk + k;
  const double2 *VVt = vv + tk * V * V;
  double *out = packed + 2 * tk * np;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
       idx < np; idx += (long long)gridDim.x * blockDim.x) {
    int col = (int)((sqrt(8.0 * (double)idx + 1.0) - 1.0) * 0.5);
    while ((long long)col * (col + 1) / 2 > idx) --col;
    while ((long long)(col + 1) * (col + 2) / 2 <= idx) ++col;
    const int row = (int)(idx - (long long)col * (col + 1) / 2);
    const double2 v = VVt[(long long)col * V + row];
    store_packed(out, idx, v);
  }
}

int launch_ortho(const DevSys &s, int nterm, const double2 *vv,
                 const double2 *cv, const double2 *cc, const double2 *s_cv,
                 double2 *y, double *packed, cudaStream_t st, bool pipe) {
  const int V = s.vale_dim, C = s.core_dim;
  if (nterm == 0) return IMAGO_OK;
  if (C == 0) {
    const long long np = (long long)V * (V + 1) / 2;
    dim3 g((unsigned)std::min<long long>((np + 255) / 256, 128), s.nk, nterm);
    k_pack_plain<<<g, 256, 0, st>>>(s, vv, packed);
    IMAGO_CUDA(cudaGetLastError());
    return IMAGO_OK;
  }
  if (pipe) {
    bool launched = false;
    const int rc = launch_ortho_pipe(s, nterm, vv, cv, cc, s_cv, packed, &launched, st);
    if (rc || launched) return rc;
  }
  const size_t smem = fused_smem(C, V);
  const int fused_y_tiles = (C + 7) / 8 * ((V + 15) / 16);
  if (smem <= kFusedMaxSmem && fused_y_tiles <= kFYTilesPerWarp * kFWarps) {
    static bool attr_set[2][64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !attr_set[s.real_k][dev]) {
      IMAGO_CUDA(cudaFuncSetAttribute(s.real_k ? k_ortho_fused<true> : k_ortho_fused<false>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kFusedMaxSmem));
      attr_set[s.real_k][dev] = true;
    }
    if (s.real_k)
      k_ortho_fused<true><<<dim3(s.nk, nterm), kFThreads, smem, st>>>(s, vv, cv, cc,
                                                                     s_cv, packed);
    else
      k_ortho_fused<false><<<dim3(s.nk, nterm), kFThreads, smem, st>>>(s, vv, cv, cc,
                                                                      s_cv, packed);
    IMAGO_CUDA(cudaGetLastError());
    return IMAGO_OK;
  }
  const int tcv = (C + kOT - 1) / kOT, tvv = (V + kOT - 1) / kOT;
  dim3 gy(tcv * tvv, s.nk, nterm);
  dim3 gw(tvv * (tvv + 1) / 2, s.nk, nterm);
  if (s.real_k) {
    k_ortho_y<true><<<gy, kOThreads, 0, st>>>(s, cv, cc, s_cv, y, 0.5);
    k_ortho_w<true><<<gw, kOThreads, 0, st>>>(s, vv, y, y, s_cv, packed, false);
  } else {
    k_ortho_y<false><<<gy, kOThreads, 0, st>>>(s, cv, cc, s_cv, y, 0.5);
    k_ortho_w<false><<<gw, kOThreads, 0, st>>>(s, vv, y, y, s_cv, packed, false);
  }
  IMAGO_CUDA(cudaGetLastError());
  return IMAGO_OK;
}

// The K-overlap phase sum (cmplxApplyPhaseFactors, intgSaving.F90:192-238;
// then kPointLatticeOriginShift): the complex contracted blocks are the
// real terms 2 axis and 2 axis + 1 of M.  One thread per (block element,
// k-point, axis), CUDA cores: the build runs once per optical run.
__global__ void __launch_bounds__(256)
    k_bloch_kov(DevSys s, DevWork w, const double *M, double2 *vv, double2 *cv,
                double2 *cc) {
  const int2 bt = w.btile[blockIdx.x];
  const DPair p = w.pairs[bt.x];
  const int ne = p.ni * p.nj, nk = s.nk;
  const int e = bt.y * kBlochCols + (threadIdx.x & (kBlochCols - 1));
  const int k = blockIdx.y * (256 / kBlochCols) + threadIdx.x / kBlochCols;
  const int ax = blockIdx.z;
  if (e >= ne || k >= nk) return;
  const double *Mr = M + (long long)(2 * ax) * w.m_total + p.moff + e;
  const double *Mi = M + (long long)(2 * ax + 1) * w.m_total + p.moff + e;
  double ar = 0.0, ai = 0.0;
  for (int u = p.ubeg; u < p.uend; ++u) {
    const long long o = (long long)(u - p.ubeg) * ne;
    const double xr = Mr[o], xi = Mi[o];
    const double2 f = s.phase[(long long)w.units[u].cell * nk + k];
    ar = ar + (f.x * xr - f.y * xi);
    ai = ai + (f.x * xi + f.y * xr);
  }
  const double *kv = s.kxyz + 3 * k;
  const double dot = kv[0] * p.L0[0] + kv[1] * p.L0[1] + kv[2] * p.L0[2];
  if (fabs(dot) >= kSmallThresh) {
    double sn, cs;
    sincos(dot, &sn, &cs);
    const double r = cs * ar - sn * ai;
    ai = cs * ai + sn * ar;
    ar = r;
  }
  const int m2 = e / p.ni, m1 = e - m2 * p.ni;
  scatter_full(s, p, (long long)ax * nk + k, m1, m2, ar, ai, vv, cv, cc);
}

int launch_bloch_kov(const DevSys &s, const DevWork &w, const double *M, double2 *vv,
                     double2 *cv, double2 *cc, cudaStream_t st) {
  if (w.nbtile == 0) return IMAGO_OK;
  if (s.nk > kBlochSmallNk) {  // the tensor-core phase sum at the tuned width
    if (w.nbtile_w == 0) return IMAGO_OK;
    dim3 grid(w.nbtile_w, (s.nk + kBK - 1) / kBK, 3);
    switch (w.bw) {
      case bloch_width(0):
        k_bloch<bloch_width(0), true><<<grid, 4 * bloch_width(0), 0, st>>>(s, w, M, vv, cv, cc);
        break;
      case bloch_width(1):
        k_bloch<bloch_width(1), true><<<grid, 4 * bloch_width(1), 0, st>>>(s, w, M, vv, cv, cc);
        break;
      case bloch_width(2):
        k_bloch<bloch_width(2), true><<<grid, 4 * bloch_width(2), 0, st>>>(s, w, M, vv, cv, cc);
        break;
      default:
        return IMAGO_ERR_INVALID;
    }
    IMAGO_CUDA(cudaGetLastError());
    return IMAGO_OK;
  }
  constexpr int kPerBlock = 256 / kBlochCols;
  dim3 grid(w.nbtile, (s.nk + kPerBlock - 1) / kPerBlock, 3);
  k_bloch_kov<<<grid, 256, 0, st>>>(s, w, M, vv, cv, cc);
  IMAGO_CUDA(cudaGetLastError());
  return IMAGO_OK;
}

__global__ void k_vv_planes(long long n, const double2 *vv, double *re, double *im) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    re[i] = vv[i].x;
    im[i] = vv[i].y;
  }
}

int launch_ortho_full(const DevSys &s, const double2 *vv, const double2 *cv,
                      const double2 *cc, const double2 *s_cv, double2 *y, double *re,
                      double *im, cudaStream_t st) {
  const int V = s.vale_dim, C = s.core_dim;
  if (C == 0) {
    const long long n = 3LL * s.nk * V * V;
    k_vv_planes<<<(unsigned)std::min<long long>((n + 255) / 256, 148 * 16), 256, 0, st>>>(
        n, vv, re, im);
    IMAGO_CUDA(cudaGetLastError());
    return IMAGO_OK;
  }
  const int tcv = (C + kOT - 1) / kOT, tvv = (V + kOT - 1) / kOT;
  k_ortho_y<false><<<dim3(tcv * tvv, s.nk, 3), kOThreads, 0, st>>>(s, cv, cc, s_cv, y, 1.0);
  IMAGO_CUDA(cudaGetLastError());
  k_ortho_w<false, true><<<dim3(tvv * tvv, s.nk, 3), kOThreads, 0, st>>>(
      s, vv, y, cv, s_cv, re, true, im);
  IMAGO_CUDA(cudaGetLastError());
  return IMAGO_OK;
}

// The orthogonalisation of a matrix whose core-core block is not Hermitian
// (the dipole matrix: <a|(r - C)|b> is not invariant under the lattice
// translation that relates a pair's two orientations).  The reference's
// sequence is applied as it stands: zher2k (VV - S^H X_cv - X_cv^H S, its
// diagonal made real), then + S^H X_cc S (makeValeVale,
// intgOrtho.F90:23-213).  With Y = X_cv - X_cc S (k_ortho_y, ycc = 1) that
// is W = VV - S^H Y - X_cv^H S, the diagonal keeping Im(S^H X_cc S):
// k_ortho_w's general form, on the tensor cores like the her2k form.
int launch_ortho_general(const DevSys &s, int nterm, const double2 *vv,
                         const double2 *cv, const double2 *cc,
                         const double2 *s_cv, double2 *y, double *packed,
                         cudaStream_t st) {
  const int V = s.vale_dim, C = s.core_dim;
  if (nterm == 0) return IMAGO_OK;
  if (C == 0) return launch_ortho(s, nterm, vv, cv, cc, s_cv, y, packed, st);
  const int tcv = (C + kOT - 1) / kOT, tvv = (V + kOT - 1) / kOT;
  k_ortho_y<false><<<dim3(tcv * tvv, s.nk, nterm), kOThreads, 0, st>>>(s, cv, cc, s_cv,
                                                                      y, 1.0);
  IMAGO_CUDA(cudaGetLastError());
  k_ortho_w<false><<<dim3(tvv * (tvv + 1) / 2, s.nk, nterm), kOThreads, 0, st>>>(
      s, vv, y, cv, s_cv, packed, true);
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
  k_split_cv<<<(unsigned)std::min<long long>((n + 255) / 256, 4096), 256, 0, st>>>(
      n, cv, re, im);
  IMAGO_CUDA(cudaGetLastError());
  return IMAGO_OK;
}

// H[q][e] += sum_t w(t, q) blk[t][e] for one or two spins q, w(t, q) =
// w[q * wstride + t] (the layout of the reference's potCoeffs(potDim, spin))
// or 1 when w is null.  Terms are added in order, so the sum is
// reproducible; each element is read once for both spins.
__global__ void k_block_axpy(const double *__restrict__ blk, int nterm,
                             long long n, const double *__restrict__ w,
                             int wstride, int spin, double *H) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    double a0 = H[e], a1 = spin > 1 ? H[n + e] : 0.0;
    for (int t = 0; t < nterm; ++t) {
      const double x = blk[t * n + e];
      a0 += (w ? __ldg(w + t) : 1.0) * x;
      if (spin > 1) a1 += (w ? __ldg(w + wstride + t) : 1.0) * x;
    }
    H[e] = a0;
    if (spin > 1) H[n + e] = a1;
  }
}

int launch_block_axpy(const double *blk, int nterm, long long n, const double *w,
                      int wstride, int spin, double *H, cudaStream_t st) {
  if (n == 0 || nterm == 0) return IMAGO_OK;
  if (spin < 1 || spin > 2) return IMAGO_ERR_INVALID;
  k_block_axpy<<<(unsigned)std::min<long long>((n + 255) / 256, 148 * 16), 256, 0, st>>>(
      blk, nterm, n, w, wstride, spin, H);
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
  k_phase<<<(unsigned)std::min<long long>((n + 255) / 256, 4096), 256, 0, st>>>(s, phase);
  IMAGO_CUDA(cudaGetLastError());
  return IMAGO_OK;
}

}  // namespace imago
