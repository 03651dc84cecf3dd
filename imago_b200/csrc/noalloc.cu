// noalloc.cu -- primitive integrals without any device allocation.
//
// imago_prim_eval copies its records to device buffers it allocates for the
// call.  Some callers cannot allow that: a process that shares its GPU
// under a fixed memory budget, or whose memory is already handed to a pool
// allocator, gets cudaMalloc failures or evictions, and a latency-bound
// loop cannot afford the device-wide synchronisation that cudaMalloc and
// cudaFree imply.  imago_prim_eval_static does the same work with its
// staging in one fixed array in device global memory, declared below, so
// it never allocates.
//
// The array is a module-scope __device__ variable: every GPU that loads
// this library holds it (IMAGO_PRIM_STATIC_BYTES) until the process exits.
// Its name is not a device address in host code, so every call takes the
// address with cudaGetSymbolAddress on the current device (cheap next to
// the copies; an address kept from an earlier call would go stale after a
// cudaDeviceReset reloads the module elsewhere).  All calls share the
// array and it keeps the last call's contents; calls that overlap on the
// GPU (from several host threads, or on several streams) would overwrite
// each other's records and must not be issued.
#include "intg.cuh"

namespace {

constexpr int kMaxRecords = IMAGO_PRIM_STATIC_MAX_RECORDS;
constexpr size_t kAlign = 256;
constexpr size_t round_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }
constexpr size_t kParamsOff = 0;
constexpr size_t kClsOff = round_up(sizeof(double) * 12 * kMaxRecords);
constexpr size_t kOutOff = kClsOff + round_up(sizeof(int) * 2 * kMaxRecords);
constexpr size_t kBytes = kOutOff + sizeof(double) * 256 * kMaxRecords;
static_assert(kBytes == IMAGO_PRIM_STATIC_BYTES,
              "IMAGO_PRIM_STATIC_BYTES must match the scratch layout");

// Records in, class pairs in, 16x16 blocks out.
static __device__ __align__(256) unsigned char g_prim_scratch[kBytes];

// Device address of g_prim_scratch on the current device, looked up on
// every call.
int scratch_address(unsigned char **out) {
  void *p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_prim_scratch);
  if (e != cudaSuccess || !p) {
    cudaGetLastError();
    return IMAGO_ERR_CUDA;
  }
  *out = static_cast<unsigned char *>(p);
  return IMAGO_OK;
}

}  // namespace

extern "C" int imago_prim_eval_static(int kind, int n, const double *params,
                                      const int *cls, double *sh) {
  if (kind < 0 || kind > 11 || n < 0 || !params || !sh) return IMAGO_ERR_INVALID;
  if (kind != 4 && !cls) return IMAGO_ERR_INVALID;
  if (n > kMaxRecords) return IMAGO_ERR_RANGE;
  if (n == 0) return IMAGO_OK;
  for (int r = 0; kind != 4 && r < n; ++r)
    if (cls[2 * r] < 0 || cls[2 * r] > 3 || cls[2 * r + 1] < 0 ||
        cls[2 * r + 1] > 3)
      return IMAGO_ERR_RANGE;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return IMAGO_ERR_NO_DEVICE;
  }
  unsigned char *base = nullptr;
  int rc = scratch_address(&base);
  if (rc) return rc;
  double *dp = reinterpret_cast<double *>(base + kParamsOff);
  int *dc = reinterpret_cast<int *>(base + kClsOff);
  double *ds = reinterpret_cast<double *>(base + kOutOff);
  // The array keeps the previous call's records: the class pairs of a Boys
  // call and the output blocks start from zero.
  if (cudaMemcpy(dp, params, sizeof(double) * 12 * n, cudaMemcpyHostToDevice) !=
      cudaSuccess)
    rc = IMAGO_ERR_CUDA;
  if (!rc) {
    const cudaError_t e =
        kind != 4 ? cudaMemcpy(dc, cls, sizeof(int) * 2 * n, cudaMemcpyHostToDevice)
                 : cudaMemset(dc, 0, sizeof(int) * 2 * n);
    if (e != cudaSuccess) rc = IMAGO_ERR_CUDA;
  }
  if (!rc && cudaMemset(ds, 0, sizeof(double) * 256 * n) != cudaSuccess)
    rc = IMAGO_ERR_CUDA;
  if (!rc) rc = imago::launch_prim_eval(kind, n, dp, dc, ds, 0);
  if (!rc && cudaMemcpy(sh, ds, sizeof(double) * 256 * n,
                        cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = IMAGO_ERR_CUDA;
  if (rc) cudaGetLastError();
  return rc;
}
