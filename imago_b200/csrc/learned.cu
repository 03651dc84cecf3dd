// learned.cu -- the learned SCF start's kernels: per-atom radial
// descriptors and a two-hidden-layer perceptron in FP32 (forward, backward,
// Adam), all written here.
//
// The network is small (tens of inputs, 128-wide hidden layers, a few
// thousand atoms per batch), so one tiled FP32 GEMM kernel (32 x 32 output
// tiles, 16 x 16 threads of 2 x 2 outputs, K staged in shared memory in
// chunks of 32) serves the forward layers, the weight gradients (A
// transposed) and the backpropagated activations (B transposed), with the
// bias, tanh and tanh-derivative epilogues fused.  Every output element is
// summed by one thread in a fixed K order, and the column sums and the
// loss by fixed-order reductions, so training is bit-reproducible.
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "intg.cuh"
#include "../../include/imago_learned.h"

namespace {

constexpr int kTile = 32;
constexpr int kTk = 32;

enum Epi { kNone = 0, kBias = 1, kBiasTanh = 2, kTanhGrad = 3 };

// C[M x N] = op(A)[M x K] op(B)[K x N]; A(m, k) = TA ? A[k lda + m] :
// A[m lda + k], B(k, n) = TB ? B[n ldb + k] : B[k ldb + n].  Epilogues:
// + bias[n]; + bias[n] then tanh; times (1 - aux[m ldc + n]^2).
template <bool TA, bool TB>
__global__ void __launch_bounds__(256)
k_gemm(int M, int N, int K, const float *__restrict__ A, int lda, const float *__restrict__ B,
       int ldb, float *__restrict__ C, int ldc, const float *__restrict__ bias, int epi,
       const float *__restrict__ aux) {
  __shared__ float sa[kTk][kTile + 1];
  __shared__ float sb[kTk][kTile + 1];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int m0 = blockIdx.y * kTile, n0 = blockIdx.x * kTile;
  float acc[2][2] = {{0.f, 0.f}, {0.f, 0.f}};
  for (int k0 = 0; k0 < K; k0 += kTk) {
    for (int q = threadIdx.x; q < kTk * kTile; q += 256) {
      const int kk = q / kTile, mm = q % kTile;
      const int m = m0 + mm, k = k0 + kk;
      sa[kk][mm] = (m < M && k < K) ? (TA ? A[(long long)k * lda + m] : A[(long long)m * lda + k])
                                    : 0.f;
      const int n = n0 + mm;
      sb[kk][mm] = (n < N && k < K) ? (TB ? B[(long long)n * ldb + k] : B[(long long)k * ldb + n])
                                    : 0.f;
    }
    __syncthreads();
#pragma unroll 8
    for (int kk = 0; kk < kTk; ++kk) {
      const float a0 = sa[kk][ty], a1 = sa[kk][ty + 16];
      const float b0 = sb[kk][tx], b1 = sb[kk][tx + 16];
      acc[0][0] = fmaf(a0, b0, acc[0][0]);
      acc[0][1] = fmaf(a0, b1, acc[0][1]);
      acc[1][0] = fmaf(a1, b0, acc[1][0]);
      acc[1][1] = fmaf(a1, b1, acc[1][1]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int m = m0 + ty + 16 * i, n = n0 + tx + 16 * j;
      if (m >= M || n >= N) continue;
      float v = acc[i][j];
      if (epi == kBias || epi == kBiasTanh) v += bias[n];
      if (epi == kBiasTanh) v = tanhf(v);
      if (epi == kTanhGrad) {
        const float a = aux[(long long)m * ldc + n];
        v *= 1.f - a * a;
      }
      C[(long long)m * ldc + n] = v;
    }
}

// out[n] = sum over rows of X [rows][cols], one thread per column, rows in
// order.
__global__ void k_colsum(const float *X, int rows, int cols, float *out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.f;
  for (int r = 0; r < rows; ++r) s += X[(long long)r * cols + c];
  out[c] = s;
}

// Masked MSE: loss = sum m (y - t)^2 / sum m and dY = 2 m (y - t) / sum m.
// One CTA of 256 threads: strided partial sums, then a fixed tree.
__global__ void k_mse(const float *y, const float *t, const float *m, long long n, float *dy,
                      float *loss) {
  __shared__ float s1[256], s2[256];
  float a = 0.f, b = 0.f;
  for (long long i = threadIdx.x; i < n; i += 256) {
    const float d = y[i] - t[i];
    a += m[i] * d * d;
    b += m[i];
  }
  s1[threadIdx.x] = a;
  s2[threadIdx.x] = b;
  __syncthreads();
  for (int h = 128; h; h >>= 1) {
    if (threadIdx.x < h) {
      s1[threadIdx.x] += s1[threadIdx.x + h];
      s2[threadIdx.x] += s2[threadIdx.x + h];
    }
    __syncthreads();
  }
  const float msum = s2[0] > 0.f ? s2[0] : 1.f;
  if (threadIdx.x == 0) *loss = s1[0] / msum;
  for (long long i = threadIdx.x; i < n; i += 256) dy[i] = 2.f * m[i] * (y[i] - t[i]) / msum;
}

__global__ void k_adam(float *p, const float *g, float *m, float *v, long long n, float lr,
                       float b1, float b2, float eps, float c1, float c2) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// Radial descriptors: one warp per atom, lane k owns descriptor k (nrad <=
// 32; more are looped), the neighbours (image-major, then atom) in order.
__global__ void k_descriptors(const double *pos, const int *species, int natoms,
                              const double *images, int nimg, double rc, int nrad, double width,
                              int nspecies, float *x) {
  const int atom = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (atom >= natoms) return;
  const int nin = nrad + nspecies;
  const double inv2w2 = 1.0 / (2.0 * width * width);
  for (int k = lane; k < nrad; k += 32) {
    const double mu = rc * (k + 1) / nrad;
    double acc = 0.0;
    for (int q = 0; q < nimg; ++q)
      for (int j = 0; j < natoms; ++j) {
        double r2 = 0.0;
        for (int c = 0; c < 3; ++c) {
          const double d = pos[3 * j + c] + images[3 * q + c] - pos[3 * atom + c];
          r2 += d * d;
        }
        if (r2 <= 0.0) continue;
        const double r = sqrt(r2);
        if (r >= rc) continue;
        const double fc = 0.5 * (cos(imago::kPi * r / rc) + 1.0);
        acc += exp(-(r - mu) * (r - mu) * inv2w2) * fc;
      }
    x[(long long)atom * nin + k] = (float)acc;
  }
  for (int s = lane; s < nspecies; s += 32)
    x[(long long)atom * nin + nrad + s] = species[atom] == s ? 1.f : 0.f;
}

template <bool TA, bool TB>
void gemm(cudaStream_t st, int M, int N, int K, const float *A, int lda, const float *B,
          int ldb, float *C, int ldc, const float *bias, int epi, const float *aux) {
  dim3 grid((N + kTile - 1) / kTile, (M + kTile - 1) / kTile);
  k_gemm<TA, TB><<<grid, 256, 0, st>>>(M, N, K, A, lda, B, ldb, C, ldc, bias, epi, aux);
}

}  // namespace

struct imago_mlp {
  int nin = 0, nh = 0, nout = 0, device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  long long np = 0;
  float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
  long long adam_t = 0;
  // activations and their gradients for the last batch
  float *h1 = nullptr, *h2 = nullptr, *y = nullptr, *dy = nullptr, *d2 = nullptr,
        *d1 = nullptr, *loss = nullptr;
  int cap = 0;
  float *w1() { return p; }
  float *b1() { return p + (long long)nin * nh; }
  float *w2() { return b1() + nh; }
  float *b2() { return w2() + (long long)nh * nh; }
  float *w3() { return b2() + nh; }
  float *b3() { return w3() + (long long)nh * nout; }
};

namespace {

int ensure(imago_mlp *c, int n) {
  if (n <= c->cap) return IMAGO_OK;
  cudaFree(c->h1);
  const long long per = 2LL * c->nh + 2LL * c->nout + 2LL * c->nh;
  void *q = nullptr;
  if (cudaMalloc(&q, sizeof(float) * (per * n + 1)) != cudaSuccess) {
    cudaGetLastError();
    c->h1 = nullptr;
    c->cap = 0;
    return IMAGO_ERR_NOMEM;
  }
  c->h1 = static_cast<float *>(q);
  c->h2 = c->h1 + (long long)c->nh * n;
  c->y = c->h2 + (long long)c->nh * n;
  c->dy = c->y + (long long)c->nout * n;
  c->d2 = c->dy + (long long)c->nout * n;
  c->d1 = c->d2 + (long long)c->nh * n;
  c->loss = c->d1 + (long long)c->nh * n;
  c->cap = n;
  return IMAGO_OK;
}

void forward(imago_mlp *c, int n, const float *x, float *y) {
  cudaStream_t st = c->stream;
  gemm<false, false>(st, n, c->nh, c->nin, x, c->nin, c->w1(), c->nh, c->h1, c->nh, c->b1(),
                     kBiasTanh, nullptr);
  gemm<false, false>(st, n, c->nh, c->nh, c->h1, c->nh, c->w2(), c->nh, c->h2, c->nh, c->b2(),
                     kBiasTanh, nullptr);
  gemm<false, false>(st, n, c->nout, c->nh, c->h2, c->nh, c->w3(), c->nout, y, c->nout,
                     c->b3(), kBias, nullptr);
}

}  // namespace

extern "C" {

int imago_mlp_create(int nin, int nh, int nout, unsigned long long seed, int device,
                     void *stream, imago_mlp **out) {
  if (!out || nin <= 0 || nh <= 0 || nout <= 0) return IMAGO_ERR_INVALID;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return IMAGO_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= ndev) return IMAGO_ERR_INVALID;
  IMAGO_CUDA(cudaSetDevice(device));
  std::unique_ptr<imago_mlp> c(new imago_mlp());
  c->nin = nin;
  c->nh = nh;
  c->nout = nout;
  c->device = device;
  c->np = (long long)nin * nh + nh + (long long)nh * nh + nh + (long long)nh * nout + nout;
  if (stream) {
    c->stream = static_cast<cudaStream_t>(stream);
  } else {
    IMAGO_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    c->own_stream = true;
  }
  void *q = nullptr;
  if (cudaMalloc(&q, sizeof(float) * 4 * c->np) != cudaSuccess) {
    cudaGetLastError();
    imago_mlp_destroy(c.release());
    return IMAGO_ERR_NOMEM;
  }
  c->p = static_cast<float *>(q);
  c->g = c->p + c->np;
  c->m = c->g + c->np;
  c->v = c->m + c->np;
  // Xavier-uniform weights from a splitmix64 stream, zero biases
  std::vector<float> h(c->np, 0.f);
  unsigned long long s = seed;
  auto next = [&]() {
    unsigned long long z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
  };
  auto fill = [&](long long off, int fan_in, int fan_out) {
    const double lim = std::sqrt(6.0 / (fan_in + fan_out));
    for (long long i = 0; i < (long long)fan_in * fan_out; ++i)
      h[off + i] = (float)((2.0 * next() - 1.0) * lim);
  };
  fill(0, nin, nh);
  fill((long long)nin * nh + nh, nh, nh);
  fill((long long)nin * nh + nh + (long long)nh * nh + nh, nh, nout);
  IMAGO_CUDA(cudaMemcpyAsync(c->p, h.data(), sizeof(float) * c->np, cudaMemcpyHostToDevice,
                             c->stream));
  IMAGO_CUDA(cudaMemsetAsync(c->m, 0, sizeof(float) * 2 * c->np, c->stream));
  IMAGO_CUDA(cudaStreamSynchronize(c->stream));
  *out = c.release();
  return IMAGO_OK;
}

void imago_mlp_destroy(imago_mlp *c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  cudaFree(c->p);
  cudaFree(c->h1);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  cudaGetLastError();
  delete c;
}

long long imago_mlp_num_params(const imago_mlp *c) { return c ? c->np : 0; }

int imago_mlp_get_params(imago_mlp *c, float *params) {
  if (!c || !params) return IMAGO_ERR_INVALID;
  IMAGO_CUDA(cudaSetDevice(c->device));
  IMAGO_CUDA(cudaMemcpyAsync(params, c->p, sizeof(float) * c->np, cudaMemcpyDeviceToHost,
                             c->stream));
  IMAGO_CUDA(cudaStreamSynchronize(c->stream));
  return IMAGO_OK;
}

int imago_mlp_set_params(imago_mlp *c, const float *params) {
  if (!c || !params) return IMAGO_ERR_INVALID;
  IMAGO_CUDA(cudaSetDevice(c->device));
  IMAGO_CUDA(cudaMemcpyAsync(c->p, params, sizeof(float) * c->np, cudaMemcpyHostToDevice,
                             c->stream));
  IMAGO_CUDA(cudaMemsetAsync(c->m, 0, sizeof(float) * 2 * c->np, c->stream));
  c->adam_t = 0;
  IMAGO_CUDA(cudaStreamSynchronize(c->stream));
  return IMAGO_OK;
}

int imago_mlp_forward(imago_mlp *c, int n, const float *x, float *y) {
  if (!c || n < 0 || (n && (!x || !y))) return IMAGO_ERR_INVALID;
  if (!n) return IMAGO_OK;
  IMAGO_CUDA(cudaSetDevice(c->device));
  int rc = ensure(c, n);
  if (rc) return rc;
  forward(c, n, x, y);
  IMAGO_CUDA(cudaGetLastError());
  return IMAGO_OK;
}

int imago_mlp_loss_grad(imago_mlp *c, int n, const float *x, const float *t, const float *mask,
                        float *loss, float *grad) {
  if (!c || n <= 0 || !x || !t || !mask || !loss) return IMAGO_ERR_INVALID;
  IMAGO_CUDA(cudaSetDevice(c->device));
  int rc = ensure(c, n);
  if (rc) return rc;
  cudaStream_t st = c->stream;
  forward(c, n, x, c->y);
  k_mse<<<1, 256, 0, st>>>(c->y, t, mask, (long long)n * c->nout, c->dy, c->loss);
  const int nin = c->nin, nh = c->nh, no = c->nout;
  float *gw1 = c->g, *gb1 = gw1 + (long long)nin * nh, *gw2 = gb1 + nh,
        *gb2 = gw2 + (long long)nh * nh, *gw3 = gb2 + nh, *gb3 = gw3 + (long long)nh * no;
  // output layer
  gemm<true, false>(st, nh, no, n, c->h2, nh, c->dy, no, gw3, no, nullptr, kNone, nullptr);
  k_colsum<<<(no + 127) / 128, 128, 0, st>>>(c->dy, n, no, gb3);
  // second hidden layer: d2 = (dy W3^T) * (1 - h2^2)
  gemm<false, true>(st, n, nh, no, c->dy, no, c->w3(), no, c->d2, nh, nullptr, kTanhGrad, c->h2);
  gemm<true, false>(st, nh, nh, n, c->h1, nh, c->d2, nh, gw2, nh, nullptr, kNone, nullptr);
  k_colsum<<<(nh + 127) / 128, 128, 0, st>>>(c->d2, n, nh, gb2);
  // first hidden layer: d1 = (d2 W2^T) * (1 - h1^2)
  gemm<false, true>(st, n, nh, nh, c->d2, nh, c->w2(), nh, c->d1, nh, nullptr, kTanhGrad, c->h1);
  gemm<true, false>(st, nin, nh, n, x, nin, c->d1, nh, gw1, nh, nullptr, kNone, nullptr);
  k_colsum<<<(nh + 127) / 128, 128, 0, st>>>(c->d1, n, nh, gb1);
  IMAGO_CUDA(cudaMemcpyAsync(loss, c->loss, sizeof(float), cudaMemcpyDeviceToHost, st));
  if (grad)
    IMAGO_CUDA(cudaMemcpyAsync(grad, c->g, sizeof(float) * c->np, cudaMemcpyDeviceToHost, st));
  IMAGO_CUDA(cudaStreamSynchronize(st));
  IMAGO_CUDA(cudaGetLastError());
  return IMAGO_OK;
}

int imago_mlp_adam_step(imago_mlp *c, float lr, float b1, float b2, float eps) {
  if (!c) return IMAGO_ERR_INVALID;
  IMAGO_CUDA(cudaSetDevice(c->device));
  c->adam_t += 1;
  const float c1 = 1.f - std::pow(b1, (float)c->adam_t);
  const float c2 = 1.f - std::pow(b2, (float)c->adam_t);
  k_adam<<<(unsigned)((c->np + 255) / 256), 256, 0, c->stream>>>(c->p, c->g, c->m, c->v, c->np,
                                                                 lr, b1, b2, eps, c1, c2);
  IMAGO_CUDA(cudaGetLastError());
  return IMAGO_OK;
}

int imago_descriptors(const double *rv, int natoms, const double *pos, const int *species,
                      int nspecies, double rc, int nrad, double width, int device, float *x) {
  if (!rv || natoms <= 0 || !pos || !species || nspecies < 1 || !(rc > 0.0) || nrad < 1 ||
      !(width > 0.0) || !x)
    return IMAGO_ERR_INVALID;
  for (int i = 0; i < natoms; ++i)
    if (species[i] < 0 || species[i] >= nspecies) return IMAGO_ERR_RANGE;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return IMAGO_ERR_NO_DEVICE;
  }
  IMAGO_CUDA(cudaSetDevice(device));
  // lattice images covering every neighbour within rc of any atom in the
  // cell: n_i up to ceil((rc + cell diagonal) / plane spacing_i)
  double rec[9], vol = 0.0;
  for (int i = 0; i < 3; ++i) {
    const int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
    for (int j = 0; j < 3; ++j) {
      const int j1 = (j + 1) % 3, j2 = (j + 2) % 3;
      rec[3 * i + j] = rv[3 * i1 + j1] * rv[3 * i2 + j2] - rv[3 * i1 + j2] * rv[3 * i2 + j1];
    }
  }
  for (int j = 0; j < 3; ++j) vol += rec[j] * rv[j];
  double diag = 0.0;
  for (int x0 = 0; x0 < 3; ++x0) {
    const double s = rv[x0] + rv[3 + x0] + rv[6 + x0];
    diag += s * s;
  }
  diag = std::sqrt(diag);
  int reps[3];
  for (int i = 0; i < 3; ++i) {
    double rl = 0.0;
    for (int j = 0; j < 3; ++j) rl += rec[3 * i + j] * rec[3 * i + j];
    const double spacing = std::fabs(vol) / std::sqrt(rl);
    reps[i] = (int)std::ceil((rc + diag) / spacing);
  }
  std::vector<double> img;
  for (int a = -reps[0]; a <= reps[0]; ++a)
    for (int b = -reps[1]; b <= reps[1]; ++b)
      for (int c = -reps[2]; c <= reps[2]; ++c)
        for (int x0 = 0; x0 < 3; ++x0) img.push_back(a * rv[x0] + b * rv[3 + x0] + c * rv[6 + x0]);
  const int nimg = (int)img.size() / 3;
  const int nin = nrad + nspecies;
  double *dpos = nullptr, *dimg = nullptr;
  int *dsp = nullptr;
  float *dx = nullptr;
  int rc_ = IMAGO_OK;
  if (cudaMalloc(&dpos, sizeof(double) * 3 * natoms) != cudaSuccess ||
      cudaMalloc(&dimg, sizeof(double) * img.size()) != cudaSuccess ||
      cudaMalloc(&dsp, sizeof(int) * natoms) != cudaSuccess ||
      cudaMalloc(&dx, sizeof(float) * (size_t)natoms * nin) != cudaSuccess)
    rc_ = IMAGO_ERR_NOMEM;
  if (!rc_ && (cudaMemcpy(dpos, pos, sizeof(double) * 3 * natoms, cudaMemcpyHostToDevice) ||
               cudaMemcpy(dimg, img.data(), sizeof(double) * img.size(),
                          cudaMemcpyHostToDevice) ||
               cudaMemcpy(dsp, species, sizeof(int) * natoms, cudaMemcpyHostToDevice)))
    rc_ = IMAGO_ERR_CUDA;
  if (!rc_) {
    k_descriptors<<<(natoms * 32 + 127) / 128, 128>>>(dpos, dsp, natoms, dimg, nimg, rc, nrad,
                                                      width, nspecies, dx);
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpy(x, dx, sizeof(float) * (size_t)natoms * nin, cudaMemcpyDeviceToHost))
      rc_ = IMAGO_ERR_CUDA;
  }
  cudaFree(dpos);
  cudaFree(dimg);
  cudaFree(dsp);
  cudaFree(dx);
  cudaGetLastError();
  return rc_;
}

}  // extern "C"
