// k_secular.cu -- the secular-equation matrices of one SCF step from the
// packed integrals (secularEqnSCF, secularEqn.F90:135-186).
//
// For each k-point the reference accumulates, in this order, the packed
// nuclear, kinetic, mass-velocity (rel = 1 only) and electronic-potential
// matrices,
//   H = NP + KE (+ MV) + sum_j w_j EP_j,
// through readPackedMatrixAccum (matrixSubs.F90:339-375), whose factor rule
// is: a factor of exactly 0.0 adds the matrix unscaled (that is how KE and
// MV are added), any other factor multiplies it -- so a potential coefficient of
// exactly zero adds its term with weight one.  It then unpacks H and the
// overlap S into the upper triangle of full matrices (unpackMatrix,
// matrixSubs.F90:405-433) for zhegv(1, 'V', 'U').  Here both triangles are
// written (the lower as the conjugate), so any Hermitian solver can take
// them, column-major [k][col][row] as the reference's valeVale.
#include <dlfcn.h>

#include <algorithm>
#include <atomic>
#include <vector>

#include <cusolverDn.h>

#include "intg.cuh"

namespace imago {
// dynamic shared memory the Jacobi kernel may take: matrices up to n = 112
constexpr size_t kJacobiMaxSmem = 216 * 1024;
namespace {

__global__ void k_secular(int V, long long np, int nk, int pot_dim,
                          const double *npm, const double *ke, const double *mv,
                          const double *ep, const double *w, const double *ol,
                          double2 *h, double2 *s) {
  const long long n = (long long)nk * np;
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < n;
       g += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(g / np);
    const long long idx = g - (long long)k * np;
    int col = (int)((sqrt(8.0 * (double)idx + 1.0) - 1.0) * 0.5);
    while ((long long)col * (col + 1) / 2 > idx) --col;
    while ((long long)(col + 1) * (col + 2) / 2 <= idx) ++col;
    const int row = (int)(idx - (long long)col * (col + 1) / 2);
    const long long pk = 2 * ((long long)k * np + idx);
    double re = npm[pk] + ke[pk], im = npm[pk + 1] + ke[pk + 1];
    if (mv) {
      re = re + mv[pk];
      im = im + mv[pk + 1];
    }
    for (int j = 0; j < pot_dim; ++j) {
      const double f = w[j] == 0.0 ? 1.0 : w[j];
      const long long pj = 2 * (((long long)j * nk + k) * np + idx);
      re = re + ep[pj] * f;
      im = im + ep[pj + 1] * f;
    }
    const long long base = (long long)k * V * V;
    h[base + (long long)col * V + row] = make_double2(re, im);
    h[base + (long long)row * V + col] = make_double2(re, -im);
    const double2 o = make_double2(ol[pk], ol[pk + 1]);
    s[base + (long long)col * V + row] = o;
    s[base + (long long)row * V + col] = make_double2(o.x, -o.y);
  }
}

// Eigenvalues of a batch of Hermitian matrices by the cyclic two-sided
// Jacobi method, one CTA per matrix held in shared memory.  Each step
// zeroes the off-diagonal entries of m/2 disjoint index pairs at once (the
// circle-method round robin over m = n rounded up to even indices, m - 1
// steps per sweep): for a_pq = |a_pq| e^{i phi},
//   tau = (a_qq - a_pp) / (2 |a_pq|),  t = sign(tau) / (|tau| + sqrt(1 + tau^2)),
//   c = 1 / sqrt(1 + t^2),  s = t c,
// and A <- J^H A J with J_pp = J_qq = c, J_pq = s e^{i phi},
// J_qp = -s e^{-i phi} (columns first, then rows).  Sweeps stop when the
// off-diagonal Frobenius norm is below 1e-14 of the whole, at most
// kJacobiMaxSweeps; the diagonal is then returned in ascending order.
// With `vec`, the rotations are also accumulated, V <- V J from V = I, in
// `vec` itself (column-major while the sweeps run, so the lanes of a warp,
// on rows, touch consecutive addresses), and at the end the columns are
// written in the order of the eigenvalues, vec[b][row][j] the row-th
// component of the j-th eigenvector (A V = V diag(w)).
constexpr int kJacobiThreads = 512;
constexpr int kJacobiMaxSweeps = 30;

__global__ void __launch_bounds__(kJacobiThreads, 1)
    k_jacobi_eigvals(int n, const double2 *a, double *w, double2 *vec) {
  extern __shared__ double2 jsm[];
  const int ld = n + 1, m = n + (n & 1), npair = m / 2;
  double2 *A = jsm;
  double *rc = reinterpret_cast<double *>(A + (size_t)n * ld);  // c, s per pair
  double2 *re = reinterpret_cast<double2 *>(rc + 2 * npair);    // e^{i phi}
  int2 *pq = reinterpret_cast<int2 *>(re + npair);
  __shared__ double red[2][kJacobiThreads / 32];
  const int tid = threadIdx.x;
  const double2 *src = a + (size_t)blockIdx.x * n * n;
  for (int i = tid; i < n * n; i += kJacobiThreads)
    A[(i / n) * ld + i % n] = src[i];
  double2 *Vt = vec ? vec + (size_t)blockIdx.x * n * n : nullptr;  // Vt[col * n + row]
  if (Vt)
    for (int i = tid; i < n * n; i += kJacobiThreads)
      Vt[i] = make_double2(i / n == i % n ? 1.0 : 0.0, 0.0);
  __syncthreads();
  for (int sweep = 0; sweep < kJacobiMaxSweeps; ++sweep) {
    // convergence: off-diagonal part of the Frobenius norm
    double off = 0.0, all = 0.0;
    for (int i = tid; i < n * n; i += kJacobiThreads) {
      const int r = i / n, c = i % n;
      const double2 v = A[r * ld + c];
      const double q = v.x * v.x + v.y * v.y;
      all += q;
      if (r != c) off += q;
    }
    for (int o = 16; o > 0; o >>= 1) {
      off += __shfl_xor_sync(0xffffffffu, off, o);
      all += __shfl_xor_sync(0xffffffffu, all, o);
    }
    if ((tid & 31) == 0) {
      red[0][tid >> 5] = off;
      red[1][tid >> 5] = all;
    }
    __syncthreads();
    off = all = 0.0;
    for (int i = 0; i < kJacobiThreads / 32; ++i) {
      off += red[0][i];
      all += red[1][i];
    }
    __syncthreads();
    if (off <= 1e-28 * all) break;
    for (int r = 0; r < m - 1; ++r) {
      if (tid < npair) {
        // circle method: index 0 stays, the others turn
        int p = 0, q = r % (m - 1) + 1;
        if (tid > 0) {
          p = (r + tid) % (m - 1) + 1;
          q = (r - tid + m - 1) % (m - 1) + 1;
        }
        if (p > q) {
          const int x = p;
          p = q;
          q = x;
        }
        double c = 1.0, sn = 0.0;
        double2 e = make_double2(1.0, 0.0);
        if (q < n) {
          const double2 apq = A[p * ld + q];
          const double mag = sqrt(apq.x * apq.x + apq.y * apq.y);
          if (mag > 1e-300) {
            e = make_double2(apq.x / mag, apq.y / mag);
            const double tau = (A[q * ld + q].x - A[p * ld + p].x) / (2.0 * mag);
            const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
            c = 1.0 / sqrt(1.0 + t * t);
            sn = t * c;
          }
        }
        pq[tid] = make_int2(p, q);
        rc[2 * tid] = c;
        rc[2 * tid + 1] = sn;
        re[tid] = e;
      }
      __syncthreads();
      // columns p, q of every row: A <- A J (a warp per pair, lanes on rows)
      for (int k = tid >> 5; k < npair; k += kJacobiThreads / 32)
      for (int row = tid & 31; row < n; row += 32) {
        const int2 x = pq[k];
        if (x.y >= n) continue;
        const double c = rc[2 * k], sn = rc[2 * k + 1];
        const double2 e = re[k];
        const double2 ap = A[row * ld + x.x], aq = A[row * ld + x.y];
        // conj(e) aq and e ap
        const double2 ceq = make_double2(e.x * aq.x + e.y * aq.y, e.x * aq.y - e.y * aq.x);
        const double2 eap = make_double2(e.x * ap.x - e.y * ap.y, e.x * ap.y + e.y * ap.x);
        A[row * ld + x.x] = make_double2(c * ap.x - sn * ceq.x, c * ap.y - sn * ceq.y);
        A[row * ld + x.y] = make_double2(sn * eap.x + c * aq.x, sn * eap.y + c * aq.y);
        if (Vt) {  // the same column rotation of V
          const double2 vp = Vt[(size_t)x.x * n + row], vq = Vt[(size_t)x.y * n + row];
          const double2 cvq = make_double2(e.x * vq.x + e.y * vq.y, e.x * vq.y - e.y * vq.x);
          const double2 evp = make_double2(e.x * vp.x - e.y * vp.y, e.x * vp.y + e.y * vp.x);
          Vt[(size_t)x.x * n + row] =
              make_double2(c * vp.x - sn * cvq.x, c * vp.y - sn * cvq.y);
          Vt[(size_t)x.y * n + row] =
              make_double2(sn * evp.x + c * vq.x, sn * evp.y + c * vq.y);
        }
      }
      __syncthreads();
      // rows p, q of every column: A <- J^H A (a warp per pair, lanes on
      // columns)
      for (int k = tid >> 5; k < npair; k += kJacobiThreads / 32)
      for (int col = tid & 31; col < n; col += 32) {
        const int2 x = pq[k];
        if (x.y >= n) continue;
        const double c = rc[2 * k], sn = rc[2 * k + 1];
        const double2 e = re[k];
        const double2 ap = A[x.x * ld + col], aq = A[x.y * ld + col];
        // e aq and conj(e) ap
        const double2 eaq = make_double2(e.x * aq.x - e.y * aq.y, e.x * aq.y + e.y * aq.x);
        const double2 cep = make_double2(e.x * ap.x + e.y * ap.y, e.x * ap.y - e.y * ap.x);
        A[x.x * ld + col] = make_double2(c * ap.x - sn * eaq.x, c * ap.y - sn * eaq.y);
        A[x.y * ld + col] = make_double2(sn * cep.x + c * aq.x, sn * cep.y + c * aq.y);
      }
      __syncthreads();
    }
  }
  // ascending order by rank (ties by index)
  double *out = w + (size_t)blockIdx.x * n;
  int *inv = reinterpret_cast<int *>(pq);  // inv[rank] = index, m >= n ints
  for (int i = tid; i < n; i += kJacobiThreads) {
    const double d = A[i * ld + i].x;
    int rank = 0;
    for (int j = 0; j < n; ++j) {
      const double dj = A[j * ld + j].x;
      rank += dj < d || (dj == d && j < i);
    }
    out[rank] = d;
    inv[rank] = i;
  }
  if (!Vt) return;
  __syncthreads();  // the diagonal is read: A's storage takes V
  for (int i = tid; i < n * n; i += kJacobiThreads) A[(i / n) * ld + i % n] = Vt[i];
  __syncthreads();
  for (int o = tid; o < n * n; o += kJacobiThreads) {
    const int row = o / n, j = o % n;
    Vt[o] = A[inv[j] * ld + row];
  }
}

}  // namespace

// ------------------------------------------------------------ traces --
// makeValenceRho's traces (valeCharge.F90:218-291): for each packed
// Hermitian matrix M_m and packed density R_s, summed over k-points,
//   matrixElementMult(M, R) = 2 sum_{off-diagonal} (Mre Rre + Mim Rim)
//                             + sum_{diagonal} Mre Rre
// (matrixSubs.F90:66-109).  One CTA per (chunk of one k-point's packed
// elements, matrix): every element is first taken as an off-diagonal one
// (contiguous loads, 32-bit indices), then the chunk's diagonal elements,
// at c (c + 3) / 2 for column c, are corrected to the diagonal weight.
// Partial sums go to part[m][k][chunk][s] and k_trace_sum adds them in
// that fixed order: the result does not
// depend on the schedule.  HBM-bound: 16 bytes of M per element and R
// from L2 when the densities fit.
constexpr int kTrThreads = 256;
constexpr int kTrPerThread = 16;
constexpr long long kTrChunk = (long long)kTrThreads * kTrPerThread;

template <int NRHO>
__global__ void __launch_bounds__(kTrThreads)
    k_packed_traces(long long np, int nk, int nchunk, const double2 *mats,
                    const double2 *rho, double *part) {
  const int m = blockIdx.y;
  const int k = blockIdx.x / nchunk, chunk = blockIdx.x - k * nchunk;
  const long long e0 = chunk * kTrChunk;
  const int len = (int)(e0 + kTrChunk < np ? kTrChunk : np - e0);
  const double2 *M = mats + ((long long)m * nk + k) * np + e0;
  const double2 *R0 = rho + (long long)k * np + e0;
  const double2 *R1 = rho + ((long long)nk + k) * np + e0;
  // every element as an off-diagonal one ...
  double a0 = 0.0, a1 = 0.0;
#pragma unroll 4
  for (int i = threadIdx.x; i < len; i += kTrThreads) {
    const double2 x = M[i], r = R0[i];
    a0 += x.x * r.x + x.y * r.y;
    if (NRHO > 1) {
      const double2 q = R1[i];
      a1 += x.x * q.x + x.y * q.y;
    }
  }
  a0 *= 2.0;
  a1 *= 2.0;
  // ... then the diagonal ones (packed index c (c + 3) / 2) of the chunk
  // corrected to Re M Re R: minus (Re M Re R + 2 Im M Im R)
  long long c = (long long)((sqrt(9.0 + 8.0 * (double)e0) - 3.0) * 0.5);
  while (c > 0 && (c - 1) * (c + 2) / 2 >= e0) --c;
  while (c * (c + 3) / 2 < e0) ++c;
  for (long long d = c + threadIdx.x; d * (d + 3) / 2 < e0 + len; d += kTrThreads) {
    const int i = (int)(d * (d + 3) / 2 - e0);
    const double2 x = M[i], r = R0[i];
    a0 -= x.x * r.x + 2.0 * x.y * r.y;
    if (NRHO > 1) {
      const double2 q = R1[i];
      a1 -= x.x * q.x + 2.0 * x.y * q.y;
    }
  }
  __shared__ double red[2][kTrThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a0 += __shfl_xor_sync(0xffffffffu, a0, o);
    a1 += __shfl_xor_sync(0xffffffffu, a1, o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][warp] = a0;
    red[1][warp] = a1;
  }
  __syncthreads();
  if (threadIdx.x < NRHO) {
    double t = 0.0;
    for (int w = 0; w < kTrThreads / 32; ++w) t += red[threadIdx.x][w];
    part[(((long long)m * nk + k) * nchunk + chunk) * NRHO + threadIdx.x] = t;
  }
}

// One warp per trace: lane l adds partials l, l + 32, ... in order, then
// the lanes' sums are combined in a fixed butterfly, so the result does not
// depend on the schedule.
__global__ void __launch_bounds__(32)
    k_trace_sum(int nrho, long long nper, const double *part, double *traces) {
  const int i = blockIdx.x, m = i / nrho, s = i - m * nrho;
  double t = 0.0;
  for (long long j = threadIdx.x; j < nper; j += 32)
    t += part[((long long)m * nper + j) * nrho + s];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  if (threadIdx.x == 0) traces[i] = t;
}

size_t packed_traces_work(int vale_dim, int nk, int nmat, int nrho) {
  const long long np = (long long)vale_dim * (vale_dim + 1) / 2;
  const long long nchunk = (np + kTrChunk - 1) / kTrChunk;
  return (size_t)nmat * nk * nchunk * nrho;
}

int launch_packed_traces(int vale_dim, int nk, int nmat, const double *mats, int nrho,
                         const double *rho, double *part, double *traces, cudaStream_t st) {
  const long long np = (long long)vale_dim * (vale_dim + 1) / 2;
  const int nchunk = (int)((np + kTrChunk - 1) / kTrChunk);
  const dim3 grid((unsigned)((long long)nk * nchunk), (unsigned)nmat);
  const double2 *m2 = reinterpret_cast<const double2 *>(mats);
  const double2 *r2 = reinterpret_cast<const double2 *>(rho);
  if (nrho > 1)
    k_packed_traces<2><<<grid, kTrThreads, 0, st>>>(np, nk, nchunk, m2, r2, part);
  else
    k_packed_traces<1><<<grid, kTrThreads, 0, st>>>(np, nk, nchunk, m2, r2, part);
  IMAGO_CUDA(cudaGetLastError());
  k_trace_sum<<<nmat * nrho, 32, 0, st>>>(nrho, (long long)nk * nchunk, part, traces);
  IMAGO_CUDA(cudaGetLastError());
  return IMAGO_OK;
}

size_t jacobi_smem(int n) {
  const int m = n + (n & 1);
  return sizeof(double2) * (size_t)n * (n + 1) + sizeof(double) * m +
         sizeof(double2) * (m / 2) + sizeof(int2) * (m / 2);
}

// ------------------------------------------ the batched library solver --
// cuSOLVER's batched Hermitian eigensolver (cusolverDnXsyevBatched, one
// call for the whole batch) is the default wherever it loads: measured on
// one B200 it takes 6.1 ms (eigenvalues) / 7.8 ms (with vectors) for 512
// matrices of n = 104, where the Jacobi kernel above takes 22.5 / 33.6 ms,
// and 150 ms for 64 matrices of n = 832 against 743 ms for one syevd per
// matrix.  It is reached through dlopen, so the library does not link
// cuSOLVER and uses the copy the process already holds; without it the
// Jacobi kernel serves n up to 112 and larger n get IMAGO_ERR_RANGE.
struct SyevApi {
  decltype(&cusolverDnCreate) create = nullptr;
  decltype(&cusolverDnSetStream) set_stream = nullptr;
  decltype(&cusolverDnCreateParams) create_params = nullptr;
  decltype(&cusolverDnXsyevBatched_bufferSize) buffer_size = nullptr;
  decltype(&cusolverDnXsyevBatched) syev = nullptr;
  bool ok = false;
};

const SyevApi &syev_api() {
  static const SyevApi api = [] {
    SyevApi a;
    void *h = dlopen("libcusolver.so.11", RTLD_NOW | RTLD_LOCAL);
    if (!h) return a;
    a.create = reinterpret_cast<decltype(a.create)>(dlsym(h, "cusolverDnCreate"));
    a.set_stream = reinterpret_cast<decltype(a.set_stream)>(dlsym(h, "cusolverDnSetStream"));
    a.create_params =
        reinterpret_cast<decltype(a.create_params)>(dlsym(h, "cusolverDnCreateParams"));
    a.buffer_size = reinterpret_cast<decltype(a.buffer_size)>(
        dlsym(h, "cusolverDnXsyevBatched_bufferSize"));
    a.syev = reinterpret_cast<decltype(a.syev)>(dlsym(h, "cusolverDnXsyevBatched"));
    a.ok = a.create && a.set_stream && a.create_params && a.buffer_size && a.syev;
    return a;
  }();
  return api;
}

// b[i] = conj(a[i]): the row-major Hermitian input read column-major is A^T
// = conj(A), so its conjugate is A in cuSOLVER's column-major layout.
__global__ void k_conj_copy(long long n, const double2 *a, double2 *b) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    b[i] = make_double2(a[i].x, -a[i].y);
}

// vec[b][row][j] = v[b][j][row]: the column-major eigenvectors to the
// row-major contract, 32 x 32 tiles through shared memory.
__global__ void k_transpose_batch(int n, const double2 *v, double2 *vec) {
  __shared__ double2 tile[32][33];
  const long long off = (long long)blockIdx.z * n * n;
  const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int row = y0 + r, col = x0 + threadIdx.x;
    if (row < n && col < n) tile[r][threadIdx.x] = v[off + (long long)row * n + col];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int row = x0 + r, col = y0 + threadIdx.x;
    if (row < n && col < n) vec[off + (long long)row * n + col] = tile[threadIdx.x][r];
  }
}

// Stream-ordered allocation from the library's pool, whose freed memory
// is kept: the solver's workspace (3 GB for 64 matrices of n = 832) is then
// not mapped again on every call.
cudaError_t pool_alloc(void **p, size_t bytes, cudaStream_t st) {
  cudaMemPool_t pool = device_scratch_pool();
  return pool ? cudaMallocFromPoolAsync(p, bytes, pool, st) : cudaMallocAsync(p, bytes, st);
}

int hermitian_eigh_batched(int n, int batch, const double2 *a, double *w, double2 *vec,
                           cudaStream_t st) {
  const SyevApi &api = syev_api();
  if (!api.ok) return IMAGO_ERR_RANGE;
  int dev = 0;
  IMAGO_CUDA(cudaGetDevice(&dev));
  // one handle per host thread and device, kept for the thread's life
  thread_local int hdev = -1;
  thread_local cusolverDnHandle_t handle = nullptr;
  thread_local cusolverDnParams_t params = nullptr;
  if (hdev != dev) {
    if (api.create(&handle) != CUSOLVER_STATUS_SUCCESS ||
        api.create_params(&params) != CUSOLVER_STATUS_SUCCESS)
      return IMAGO_ERR_CUDA;
    hdev = dev;
  }
  if (api.set_stream(handle, st) != CUSOLVER_STATUS_SUCCESS) return IMAGO_ERR_CUDA;
  const long long elems = (long long)n * n * batch;
  const cusolverEigMode_t jobz = vec ? CUSOLVER_EIG_MODE_VECTOR : CUSOLVER_EIG_MODE_NOVECTOR;
  double2 *work = nullptr;
  int *info = nullptr;
  void *dbuf = nullptr;
  int rc = IMAGO_OK;
  size_t dws = 0, hws = 0;
  std::vector<char> hbuf;
  if (pool_alloc(reinterpret_cast<void **>(&work), elems * sizeof(double2), st) !=
          cudaSuccess ||
      pool_alloc(reinterpret_cast<void **>(&info), batch * sizeof(int), st) != cudaSuccess) {
    cudaGetLastError();
    rc = IMAGO_ERR_NOMEM;
  }
  if (!rc) {
    k_conj_copy<<<(unsigned)std::min<long long>((elems + 255) / 256, 148 * 16), 256, 0, st>>>(
        elems, a, work);
    if (cudaGetLastError() != cudaSuccess) rc = IMAGO_ERR_CUDA;
  }
  if (!rc && api.buffer_size(handle, params, jobz, CUBLAS_FILL_MODE_LOWER, n, CUDA_C_64F, work,
                             n, CUDA_R_64F, w, CUDA_C_64F, &dws, &hws,
                             batch) != CUSOLVER_STATUS_SUCCESS)
    rc = IMAGO_ERR_CUDA;
  if (!rc && pool_alloc(&dbuf, dws ? dws : 16, st) != cudaSuccess) {
    cudaGetLastError();
    rc = IMAGO_ERR_NOMEM;
  }
  if (!rc) hbuf.resize(hws ? hws : 16);
  if (!rc && api.syev(handle, params, jobz, CUBLAS_FILL_MODE_LOWER, n, CUDA_C_64F, work, n,
                      CUDA_R_64F, w, CUDA_C_64F, dbuf, dws, hbuf.data(), hws, info,
                      batch) != CUSOLVER_STATUS_SUCCESS)
    rc = IMAGO_ERR_CUDA;
  if (!rc && vec) {
    const dim3 grid((n + 31) / 32, (n + 31) / 32, batch);
    k_transpose_batch<<<grid, dim3(32, 8), 0, st>>>(n, work, vec);
    if (cudaGetLastError() != cudaSuccess) rc = IMAGO_ERR_CUDA;
  }
  std::vector<int> hinfo(batch, 0);
  if (!rc && (cudaMemcpyAsync(hinfo.data(), info, batch * sizeof(int), cudaMemcpyDeviceToHost,
                              st) != cudaSuccess ||
              cudaStreamSynchronize(st) != cudaSuccess))
    rc = IMAGO_ERR_CUDA;
  for (int b = 0; b < batch && !rc; ++b)
    if (hinfo[b] != 0) rc = IMAGO_ERR_CUDA;  // not converged or an invalid argument
  if (dbuf) cudaFreeAsync(dbuf, st);
  if (info) cudaFreeAsync(info, st);
  if (work) cudaFreeAsync(work, st);
  cudaGetLastError();
  return rc;
}

}  // namespace imago

namespace {
// 0: the batched library solver where it loads, else the Jacobi kernel;
// 1: the Jacobi kernel up to n = 112; 2: the batched library solver only
std::atomic<int> g_eig_solver{0};
}  // namespace

extern "C" int imago_hermitian_set_solver(int mode) {
  if (mode < 0 || mode > 2) return IMAGO_ERR_INVALID;
  g_eig_solver.store(mode);
  return IMAGO_OK;
}

extern "C" int imago_hermitian_solver(int *mode) {
  if (!mode) return IMAGO_ERR_INVALID;
  *mode = g_eig_solver.load();
  return IMAGO_OK;
}

extern "C" int imago_hermitian_eigh(int n, int batch, const double *a, double *w,
                                    double *vec, void *stream) {
  if (n <= 0 || batch < 0 || !a || !w) return IMAGO_ERR_INVALID;
  if (batch == 0) return IMAGO_OK;
  const size_t smem = imago::jacobi_smem(n);
  const int mode = g_eig_solver.load();
  if (smem > imago::kJacobiMaxSmem || mode == 2 || (mode == 0 && imago::syev_api().ok))
    return imago::hermitian_eigh_batched(n, batch, reinterpret_cast<const double2 *>(a), w,
                                         reinterpret_cast<double2 *>(vec),
                                         (cudaStream_t)stream);
  static bool attr_set[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return IMAGO_ERR_NO_DEVICE;
  }
  if (dev >= 0 && dev < 64 && !attr_set[dev]) {
    if (cudaFuncSetAttribute(imago::k_jacobi_eigvals,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)imago::kJacobiMaxSmem) != cudaSuccess) {
      cudaGetLastError();
      return IMAGO_ERR_CUDA;
    }
    attr_set[dev] = true;
  }
  imago::k_jacobi_eigvals<<<batch, imago::kJacobiThreads, smem, (cudaStream_t)stream>>>(
      n, reinterpret_cast<const double2 *>(a), w, reinterpret_cast<double2 *>(vec));
  if (cudaGetLastError() != cudaSuccess) return IMAGO_ERR_CUDA;
  return IMAGO_OK;
}

extern "C" int imago_hermitian_eigvals(int n, int batch, const double *a,
                                       double *w, void *stream) {
  return imago_hermitian_eigh(n, batch, a, w, nullptr, stream);
}

extern "C" int imago_secular_matrices_rel(int vale_dim, int num_kpoints, int pot_dim,
                                          const double *np_packed,
                                          const double *ke_packed,
                                          const double *mv_packed,
                                          const double *ep_packed,
                                          const double *pot_coeffs,
                                          const double *ol_packed, double *h_full,
                                          double *s_full, void *stream) {
  if (vale_dim <= 0 || num_kpoints <= 0 || pot_dim < 0 || !np_packed ||
      !ke_packed || (pot_dim > 0 && (!ep_packed || !pot_coeffs)) || !ol_packed ||
      !h_full || !s_full)
    return IMAGO_ERR_INVALID;
  const long long np = (long long)vale_dim * (vale_dim + 1) / 2;
  const long long n = np * num_kpoints;
  const unsigned grid = (unsigned)std::min<long long>((n + 255) / 256, 148 * 16);
  imago::k_secular<<<grid, 256, 0, (cudaStream_t)stream>>>(
      vale_dim, np, num_kpoints, pot_dim, np_packed, ke_packed, mv_packed, ep_packed,
      pot_coeffs, ol_packed, reinterpret_cast<double2 *>(h_full),
      reinterpret_cast<double2 *>(s_full));
  if (cudaGetLastError() != cudaSuccess) return IMAGO_ERR_CUDA;
  return IMAGO_OK;
}

extern "C" int imago_secular_matrices(int vale_dim, int num_kpoints, int pot_dim,
                                      const double *np_packed,
                                      const double *ke_packed,
                                      const double *ep_packed,
                                      const double *pot_coeffs,
                                      const double *ol_packed, double *h_full,
                                      double *s_full, void *stream) {
  return imago_secular_matrices_rel(vale_dim, num_kpoints, pot_dim, np_packed,
                                    ke_packed, nullptr, ep_packed, pot_coeffs,
                                    ol_packed, h_full, s_full, stream);
}
