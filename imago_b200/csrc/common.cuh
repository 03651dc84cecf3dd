// common.cuh -- shared constants, class tables and error handling for the
// B200 integral setup.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

#include "../../include/imago_intg.h"

namespace imago {

constexpr double kPi = 3.141592653589793;   // constants.f90:36
constexpr double kSmallThresh = 1.0e-8;     // constants.f90:49
constexpr double kPackThresh = 1.0e-10;     // intgOrtho.F90:138-139

// Number of real-solid-harmonic functions of a class l (all functions up
// to l, as lmAlphaIndex classes them: basis.f90:138-146) and the number of
// Cartesian components behind them.
__host__ __device__ constexpr int nsh(int l) { return (l + 1) * (l + 1); }
__host__ __device__ constexpr int ncart(int l) {
  return (l + 1) * (l + 2) * (l + 3) / 6;
}
// Number of Hermite triples (t,u,v) with t+u+v <= L.
__host__ __device__ constexpr int nherm(int L) {
  return (L + 1) * (L + 2) * (L + 3) / 6;
}

// Cartesian components in the reference's pc order (gaussIntegrals.f90
// header comment: 1 s; 2 x; 3 y; 4 z; 5 xx; 6 yy; 7 zz; 8 xy; 9 xz; 10 yz;
// 11 xyz; 12 xxy; 13 xxz; 14 yyx; 15 yyz; 16 zzx; 17 zzy; 18 xxx; 19 yyy;
// 20 zzz), as exponent triples.
__host__ __device__ constexpr int cart_exp(int p, int axis) {
  constexpr int t[20][3] = {
      {0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0}, {0, 2, 0},
      {0, 0, 2}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}, {2, 1, 0},
      {2, 0, 1}, {1, 2, 0}, {0, 2, 1}, {1, 0, 2}, {0, 1, 2}, {3, 0, 0},
      {0, 3, 0}, {0, 0, 3}};
  return t[p][axis];
}

// Real-solid-harmonic component -> Cartesian combination, the reference's
// sh order (1 s; 2 x; 3 y; 4 z; 5 xy; 6 xz; 7 yz; 8 xx-yy; 9 2zz-xx-yy;
// 10 xyz; 11 xxz-yyz; 12 xxx-3yyx; 13 3xxy-yyy; 14 2zzz-3xxz-3yyz;
// 15 4zzx-xxx-yyx; 16 4zzy-xxy-yyy; src/scripts/osrecurintg.py:332-426).
__host__ __device__ constexpr int sh_nterm(int s) {
  constexpr int n[16] = {1, 1, 1, 1, 1, 1, 1, 2, 3, 1, 2, 2, 2, 3, 3, 3};
  return n[s];
}
__host__ __device__ constexpr int sh_cart(int s, int k) {
  constexpr int p[16][3] = {{0, 0, 0},    {1, 0, 0},    {2, 0, 0},
                            {3, 0, 0},    {7, 0, 0},    {8, 0, 0},
                            {9, 0, 0},    {4, 5, 0},    {6, 4, 5},
                            {10, 0, 0},   {12, 14, 0},  {17, 13, 0},
                            {11, 18, 0},  {19, 12, 14}, {15, 17, 13},
                            {16, 11, 18}};
  return p[s][k];
}
__host__ __device__ constexpr double sh_coef(int s, int k) {
  constexpr double c[16][3] = {{1, 0, 0},   {1, 0, 0},   {1, 0, 0},
                               {1, 0, 0},   {1, 0, 0},   {1, 0, 0},
                               {1, 0, 0},   {1, -1, 0},  {2, -1, -1},
                               {1, 0, 0},   {1, -1, 0},  {1, -3, 0},
                               {3, -1, 0},  {2, -3, -3}, {4, -1, -1},
                               {4, -1, -1}};
  return c[s][k];
}

// Index of Hermite triple (t,u,v), t+u+v <= L, in a packed list ordered by
// total order n = t+u+v, then t descending, then u descending.
__host__ __device__ constexpr int herm_index(int t, int u, int v) {
  int n = t + u + v;
  int base = n * (n + 1) * (n + 2) / 6;        // triples of lower order
  int r = n - t;                               // u + v
  int off = (n - t) * (n - t + 1) / 2;         // earlier t at this order
  return base + off + (r - u);
}

}  // namespace imago

#define IMAGO_CUDA(call)                                                   \
  do {                                                                     \
    cudaError_t e_ = (call);                                               \
    if (e_ != cudaSuccess) {                                               \
      std::fprintf(stderr, "imago: CUDA error %s at %s:%d\n",              \
                   cudaGetErrorString(e_), __FILE__, __LINE__);            \
      return IMAGO_ERR_CUDA;                                               \
    }                                                                      \
  } while (0)
