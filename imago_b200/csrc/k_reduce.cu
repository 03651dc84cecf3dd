// k_reduce.cu -- the Cholesky reduction of the generalised Hermitian
// problem H c = E S c of one SCF step, the back-transformation of its
// eigenvectors and the packed valence density, for every k-point at once.
//
// The reference hands each k-point's pair to LAPACK zhegv(1, 'V', 'U')
// (solveZHEGV, interfaces.F90:73-120): zpotrf factors S = U^H U, zhegst
// forms inv(U^H) H inv(U), zheev diagonalises it, and ztrsm takes the
// vectors back, c = inv(U) y.  Here the same factor is kept as L = U^H
// (from S's lower triangle, which is the conjugate of its upper one), and
// A = L^-1 H L^-H is formed by two forward substitutions,
//   Y = L^-1 H,  A = L^-1 Y^H  (H = H^H, so Y^H = H L^-H),
// one CTA per k-point with L in shared memory (column-packed, n up to 128).
// zpotrf's failure rule is kept: a pivot that is not positive (or is NaN)
// stops the factorisation and is reported as the order of that leading
// minor.
//
// The density of makeValenceRho (valeCharge.F90:181-192) is a sequence of
// zher updates rho <- rho + f_j c_j c_j^H over the occupied states, upper
// triangle, diagonal kept real; the kernel here forms each packed element
// as the same sum in the same state order, a CTA per 32 x 32 tile of the
// upper triangle of one k-point.
#include <algorithm>

#include "intg.cuh"

namespace imago {
namespace {

constexpr int kRedThreads = 256;
constexpr int kRedWarps = kRedThreads / 32;
constexpr int kRedMaxN = 128;  // 4 rows per lane in the substitutions
constexpr int kRedCols = 4;    // right-hand sides a warp carries at once

// Column-packed lower storage: L(r, j), r >= j, at pcol(n, j) + r - j.
__device__ __forceinline__ int pcol(int n, int j) { return j * n - (j * (j - 1)) / 2; }

// c - a b
__device__ __forceinline__ double2 csub_mul(double2 c, double2 a, double2 b) {
  return make_double2(fma(-a.x, b.x, fma(a.y, b.y, c.x)), fma(-a.x, b.y, fma(-a.y, b.x, c.y)));
}
// c - a conj(b)
__device__ __forceinline__ double2 csub_mulc(double2 c, double2 a, double2 b) {
  return make_double2(fma(-a.x, b.x, fma(-a.y, b.y, c.x)), fma(-a.y, b.x, fma(a.x, b.y, c.y)));
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

__device__ __forceinline__ double2 shfl2(double2 v, int l) {
  return make_double2(__shfl_sync(0xffffffffu, v.x, l), __shfl_sync(0xffffffffu, v.y, l));
}

// The pivot of column q, whose update is complete (the calling warp made
// it): L_qq = sqrt(a_qq) and the rows below scaled by its reciprocal, as
// zpotf2 scales by 1 / ajj, which linv[q] keeps for the substitutions.
// False on every lane when a_qq is not positive.
__device__ __forceinline__ bool pivot_column(double2 *Lp, double *linv, int n, int q,
                                             int lane) {
  const int pq = pcol(n, q) - q;
  const double d = Lp[pq + q].x;
  if (!(d > 0.0)) return false;
  const double sd = sqrt(d), inv = 1.0 / sd;
  __syncwarp();
  for (int r = q + 1 + lane; r < n; r += 32) {
    const double2 v = Lp[pq + r];
    Lp[pq + r] = make_double2(v.x * inv, v.y * inv);
  }
  if (lane == 0) {
    Lp[pq + q] = make_double2(sd, 0.0);
    linv[q] = inv;
  }
  return true;
}

// Forward substitution L x = b for NC right-hand sides carried by one
// warp, row r = lane + 32 m in w[c][m] (zero beyond n).  Column form, as
// ztrsm('L', 'L', 'N', 'N') runs it, but with x_j = b_j (1 / L_jj) (a
// multiplication where ztrsm divides: the division sat on the critical
// path of every step), then b_r <- b_r - L_rj x_j for r > j.  Each step
// waits on the previous one through one lane's row, so a warp carries
// several right-hand sides to have independent work in flight.
template <int M, int NC>
__device__ __forceinline__ void lower_solve(const double2 *Lp, const double *linv, int n,
                                            double2 (&w)[NC][M], int lane) {
#pragma unroll
  for (int m = 0; m < M; ++m) {
    for (int l = 0; l < 32; ++l) {
      const int j = 32 * m + l;
      if (j >= n) break;
      const double dj = linv[j];
      const int pj = pcol(n, j) - j;
      double2 x[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const double2 b = shfl2(w[c][m], l);
        x[c] = make_double2(b.x * dj, b.y * dj);
        if (lane == l) w[c][m] = x[c];
      }
#pragma unroll
      for (int mm = m; mm < M; ++mm) {
        const int r = lane + 32 * mm;
        if (r > j && r < n) {
          const double2 lr = Lp[pj + r];
#pragma unroll
          for (int c = 0; c < NC; ++c) w[c][mm] = csub_mul(w[c][mm], lr, x[c]);
        }
      }
    }
  }
}

// Backward substitution L^H x = b (the upper factor U = L^H of zpotrf), L
// row-packed: L(j, i), i <= j, at j (j + 1) / 2 + i.  Column form, as
// ztrsm('L', 'U', 'N', 'N') runs it (again multiplying by 1 / L_jj): x_j
// from the last row up, then b_r <- b_r - conj(L_jr) x_j for r < j.
template <int M, int NC>
__device__ __forceinline__ void upper_solve(const double2 *Lr, const double *linv, int n,
                                            double2 (&w)[NC][M], int lane) {
#pragma unroll
  for (int m = M - 1; m >= 0; --m) {
    for (int l = 31; l >= 0; --l) {
      const int j = 32 * m + l;
      if (j >= n) continue;
      const double dj = linv[j];
      const int rj = j * (j + 1) / 2;
      double2 x[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const double2 b = shfl2(w[c][m], l);
        x[c] = make_double2(b.x * dj, b.y * dj);
        if (lane == l) w[c][m] = x[c];
      }
#pragma unroll
      for (int mm = 0; mm <= m; ++mm) {
        const int r = lane + 32 * mm;
        if (r < j) {
          const double2 lc = cconj(Lr[rj + r]);
#pragma unroll
          for (int c = 0; c < NC; ++c) w[c][mm] = csub_mul(w[c][mm], lc, x[c]);
        }
      }
    }
  }
}

size_t reduce_smem(int n) {
  const size_t np = (size_t)n * (n + 1) / 2;
  return np * sizeof(double2) + ((size_t)n * sizeof(double) + 15) / 16 * 16;
}

// One CTA per k-point: S's lower triangle into shared memory, the
// right-looking Cholesky factorisation (the warp that updates column j + 1
// also takes its pivot, so one barrier per column), then Y = L^-1 H column
// by column, stored as Y^H, and A = L^-1 Y^H in place.  h and s are
// column-major per k-point (H(r, c) at c n + r, both triangles, as
// imago_secular_matrices writes them); a receives A row-major (stored as
// conj(A(r, c)) at c n + r, which is A(c, r) for the Hermitian A).  info[k]
// is zpotrf's: 0, or the order of the first leading minor of S that is not
// positive definite (A is then zero).
template <int M>
__global__ void __launch_bounds__(kRedThreads, 2)
    k_secular_reduce(int n, const double2 *h, const double2 *s, double2 *a, double2 *lfac,
                     int *info) {
  extern __shared__ __align__(16) unsigned char rsm[];
  const int np = n * (n + 1) / 2;
  double2 *Lp = reinterpret_cast<double2 *>(rsm);
  double *linv = reinterpret_cast<double *>(Lp + np);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long long base = (long long)blockIdx.x * n * n;
  // column j of S from row j down is contiguous in both layouts
  for (int j = warp; j < n; j += kRedWarps) {
    const int pj = pcol(n, j) - j;
    for (int r = j + lane; r < n; r += 32) Lp[pj + r] = s[base + (long long)j * n + r];
  }
  __syncthreads();
  int failed = 0;  // 1 + the failing pivot, on the lanes of the warp that met it
  if (warp == 0 && !pivot_column(Lp, linv, n, 0, lane)) failed = 1;
  bool stop = __syncthreads_or(failed);
  for (int j = 0; j + 1 < n && !stop; ++j) {
    const int pj = pcol(n, j) - j;
    // columns q > j: A(r, q) -= L(r, j) conj(L(q, j)), r >= q; a lane's
    // rows (at most M, n <= 32 M) loaded together so that their updates
    // overlap
    for (int q = j + 1 + warp; q < n; q += kRedWarps) {
      const double2 lq = Lp[pj + q];
      const int pq = pcol(n, q) - q;
      double2 av[M], lv[M];
#pragma unroll
      for (int m = 0; m < M; ++m) {
        const int r = q + lane + 32 * m;
        if (r < n) {
          av[m] = Lp[pq + r];
          lv[m] = Lp[pj + r];
        }
      }
#pragma unroll
      for (int m = 0; m < M; ++m) {
        const int r = q + lane + 32 * m;
        if (r < n) Lp[pq + r] = csub_mulc(av[m], lv[m], lq);
      }
      if (q == j + 1) {
        __syncwarp();
        if (!pivot_column(Lp, linv, n, q, lane)) failed = q + 1;
      }
    }
    stop = __syncthreads_or(failed);
  }
  if (stop) {
    if (failed && lane == 0 && info) info[blockIdx.x] = failed;
    for (int t = tid; t < n * n; t += kRedThreads) a[base + t] = make_double2(0.0, 0.0);
    return;
  }
  if (tid == 0 && info) info[blockIdx.x] = 0;
  if (lfac)
    for (int t = tid; t < np; t += kRedThreads) lfac[(long long)blockIdx.x * np + t] = Lp[t];
  constexpr int NC = kRedCols;
  // Y = L^-1 H: column c of H in, conj(Y(r, c)) out at r n + c
  for (int c0 = warp * NC; c0 < n; c0 += kRedWarps * NC) {
    double2 w[NC][M];
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
      for (int m = 0; m < M; ++m) {
        const int r = lane + 32 * m, col = c0 + c;
        w[c][m] = (r < n && col < n) ? h[base + (long long)col * n + r] : make_double2(0.0, 0.0);
      }
    lower_solve<M, NC>(Lp, linv, n, w, lane);
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
      for (int m = 0; m < M; ++m) {
        const int r = lane + 32 * m, col = c0 + c;
        if (r < n && col < n) a[base + (long long)r * n + col] = cconj(w[c][m]);
      }
  }
  __syncthreads();  // Y^H complete (global writes of this CTA visible to it)
  // A = L^-1 Y^H: each warp reads its columns whole before replacing them
  for (int c0 = warp * NC; c0 < n; c0 += kRedWarps * NC) {
    double2 w[NC][M];
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
      for (int m = 0; m < M; ++m) {
        const int r = lane + 32 * m, col = c0 + c;
        w[c][m] = (r < n && col < n) ? a[base + (long long)col * n + r] : make_double2(0.0, 0.0);
      }
    lower_solve<M, NC>(Lp, linv, n, w, lane);
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
      for (int m = 0; m < M; ++m) {
        const int r = lane + 32 * m, col = c0 + c;
        if (r < n && col < n) a[base + (long long)col * n + r] = cconj(w[c][m]);
      }
  }
}

// One CTA per k-point: c = L^-H y for the first ns eigenvectors, y in
// vec[k][row][j] (the layout imago_hermitian_eigh writes), c state-major:
// c[k][j][row].
template <int M>
__global__ void __launch_bounds__(kRedThreads, 2)
    k_secular_back(int n, int ns, const double2 *lfac, const double2 *vec, double2 *out) {
  extern __shared__ __align__(16) unsigned char rsm[];
  const int np = n * (n + 1) / 2;
  double2 *Lr = reinterpret_cast<double2 *>(rsm);
  double *linv = reinterpret_cast<double *>(Lr + np);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const double2 *lk = lfac + (long long)blockIdx.x * np;
  for (int j = warp; j < n; j += kRedWarps) {
    const int pj = pcol(n, j) - j;
    for (int r = j + lane; r < n; r += 32) Lr[r * (r + 1) / 2 + j] = lk[pj + r];
    if (lane == 0) linv[j] = 1.0 / lk[pj + j].x;
  }
  __syncthreads();
  const long long vbase = (long long)blockIdx.x * n * n;
  const long long obase = (long long)blockIdx.x * ns * n;
  constexpr int NC = kRedCols;
  for (int c0 = warp * NC; c0 < ns; c0 += kRedWarps * NC) {
    double2 w[NC][M];
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
      for (int m = 0; m < M; ++m) {
        const int r = lane + 32 * m, col = c0 + c;
        w[c][m] = (r < n && col < ns) ? vec[vbase + (long long)r * n + col] : make_double2(0.0, 0.0);
      }
    upper_solve<M, NC>(Lr, linv, n, w, lane);
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
      for (int m = 0; m < M; ++m) {
        const int r = lane + 32 * m, col = c0 + c;
        if (r < n && col < ns) out[obase + (long long)col * n + r] = w[c][m];
      }
  }
}

// rho(r, q) = sum_j f_j c_j(r) conj(c_j(q)) for r <= q of one 32 x 32 tile
// (row tile I <= column tile J, blockIdx.x over the pairs) of k-point
// blockIdx.y, the states in order, 32 at a time through shared memory: each
// term as zher adds it, x(r) * (f conj(x(q))), the diagonal kept real.
// c is state-major, c[k][j][r] (ld_states states per k-point, the first ns
// used); f[k][j]; rho packed as packMatrix leaves it, (r, q) at
// q (q + 1) / 2 + r.
constexpr int kPdThreads = 256;
constexpr int kPdStates = 32;

__global__ void __launch_bounds__(kPdThreads)
    k_packed_density(int n, int ld_states, int ns, const double2 *c, const double *f,
                     double2 *rho) {
  __shared__ double2 crow[kPdStates][32], ccol[kPdStates][32];
  int J = (int)((sqrt(8.0 * blockIdx.x + 1.0) - 1.0) * 0.5);
  while (J * (J + 1) / 2 > (int)blockIdx.x) --J;
  while ((J + 1) * (J + 2) / 2 <= (int)blockIdx.x) ++J;
  const int I = (int)blockIdx.x - J * (J + 1) / 2;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int k = blockIdx.y, r0 = 32 * I, q0 = 32 * J;
  const double2 *ck = c + (long long)k * ld_states * n;
  const double *fk = f + (long long)k * ld_states;
  double2 acc[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) acc[i] = make_double2(0.0, 0.0);
  for (int s0 = 0; s0 < ns; s0 += kPdStates) {
    for (int t = tid; t < kPdStates * 32; t += kPdThreads) {
      const int js = t >> 5, e = t & 31, j = s0 + js;
      double2 u = make_double2(0.0, 0.0), v = u;
      if (j < ns) {
        const double fj = fk[j];
        if (r0 + e < n) u = ck[(long long)j * n + r0 + e];
        if (q0 + e < n) {
          const double2 x = ck[(long long)j * n + q0 + e];
          v = make_double2(fj * x.x, -fj * x.y);
        }
      }
      crow[js][e] = u;
      ccol[js][e] = v;
    }
    __syncthreads();
    const int jn = min(kPdStates, ns - s0);
    for (int js = 0; js < jn; ++js) {
      const double2 u = crow[js][lane];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const double2 v = ccol[js][warp + 8 * i];
        acc[i].x = fma(u.x, v.x, fma(-u.y, v.y, acc[i].x));
        acc[i].y = fma(u.x, v.y, fma(u.y, v.x, acc[i].y));
      }
    }
    __syncthreads();
  }
  const int r = r0 + lane;
  double2 *rk = rho + (long long)k * ((long long)n * (n + 1) / 2);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int q = q0 + warp + 8 * i;
    if (q < n && r <= q) {
      double2 v = acc[i];
      if (r == q) v.y = 0.0;
      rk[(long long)q * (q + 1) / 2 + r] = v;
    }
  }
}

template <typename K>
int set_smem_once(K kernel, int idx, size_t bytes) {
  static bool done[8][64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return IMAGO_ERR_NO_DEVICE;
  }
  if (dev < 0 || dev >= 64 || !done[idx][dev]) {
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) !=
        cudaSuccess) {
      cudaGetLastError();
      return IMAGO_ERR_CUDA;
    }
    if (dev >= 0 && dev < 64) done[idx][dev] = true;
  }
  return IMAGO_OK;
}

}  // namespace
}  // namespace imago

using imago::kRedMaxN;

extern "C" int imago_secular_reduce(int n, int num_kpoints, const double *h_full,
                                    const double *s_full, double *a, double *l_packed,
                                    int *info, void *stream) {
  if (n <= 0 || num_kpoints < 0 || !h_full || !s_full || !a || h_full == a || s_full == a)
    return IMAGO_ERR_INVALID;
  if (n > kRedMaxN) return IMAGO_ERR_RANGE;
  if (num_kpoints == 0) return IMAGO_OK;
  const int M = (n + 31) / 32;
  const size_t smem = imago::reduce_smem(n), cap = imago::reduce_smem(kRedMaxN);
  auto go = [&](auto kernel, int idx) {
    const int rc = imago::set_smem_once(kernel, idx, cap);
    if (rc) return rc;
    kernel<<<num_kpoints, imago::kRedThreads, smem, (cudaStream_t)stream>>>(
        n, reinterpret_cast<const double2 *>(h_full), reinterpret_cast<const double2 *>(s_full),
        reinterpret_cast<double2 *>(a), reinterpret_cast<double2 *>(l_packed), info);
    return cudaGetLastError() == cudaSuccess ? (int)IMAGO_OK : (int)IMAGO_ERR_CUDA;
  };
  switch (M) {
    case 1: return go(imago::k_secular_reduce<1>, 0);
    case 2: return go(imago::k_secular_reduce<2>, 1);
    case 3: return go(imago::k_secular_reduce<3>, 2);
    default: return go(imago::k_secular_reduce<4>, 3);
  }
}

extern "C" int imago_secular_back(int n, int num_kpoints, int num_states, const double *l_packed,
                                  const double *vec, double *c, void *stream) {
  if (n <= 0 || num_kpoints < 0 || num_states < 0 || num_states > n || !l_packed || !vec || !c)
    return IMAGO_ERR_INVALID;
  if (n > kRedMaxN) return IMAGO_ERR_RANGE;
  if (num_kpoints == 0 || num_states == 0) return IMAGO_OK;
  const int M = (n + 31) / 32;
  const size_t smem = imago::reduce_smem(n), cap = imago::reduce_smem(kRedMaxN);
  auto go = [&](auto kernel, int idx) {
    const int rc = imago::set_smem_once(kernel, idx, cap);
    if (rc) return rc;
    kernel<<<num_kpoints, imago::kRedThreads, smem, (cudaStream_t)stream>>>(
        n, num_states, reinterpret_cast<const double2 *>(l_packed),
        reinterpret_cast<const double2 *>(vec), reinterpret_cast<double2 *>(c));
    return cudaGetLastError() == cudaSuccess ? (int)IMAGO_OK : (int)IMAGO_ERR_CUDA;
  };
  switch (M) {
    case 1: return go(imago::k_secular_back<1>, 4);
    case 2: return go(imago::k_secular_back<2>, 5);
    case 3: return go(imago::k_secular_back<3>, 6);
    default: return go(imago::k_secular_back<4>, 7);
  }
}

extern "C" int imago_packed_density(int n, int num_kpoints, int ld_states, int num_states,
                                    const double *c, const double *population, double *rho,
                                    void *stream) {
  if (n <= 0 || num_kpoints < 0 || num_states < 0 || ld_states < num_states || !c ||
      !population || !rho)
    return IMAGO_ERR_INVALID;
  if (num_kpoints == 0) return IMAGO_OK;
  const int nt = (n + 31) / 32;
  if (num_kpoints > 65535) return IMAGO_ERR_RANGE;
  const dim3 grid((unsigned)(nt * (nt + 1) / 2), (unsigned)num_kpoints);
  imago::k_packed_density<<<grid, imago::kPdThreads, 0, (cudaStream_t)stream>>>(
      n, ld_states, num_states, reinterpret_cast<const double2 *>(c), population,
      reinterpret_cast<double2 *>(rho));
  return cudaGetLastError() == cudaSuccess ? (int)IMAGO_OK : (int)IMAGO_ERR_CUDA;
}
