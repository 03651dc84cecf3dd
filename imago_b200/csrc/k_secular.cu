// k_secular.cu -- the secular-equation matrices of one SCF step from the
// packed integrals (secularEqnSCF, secularEqn.F90:135-186).
//
// For each k-point the reference accumulates, in this order, the packed
// nuclear, kinetic and electronic-potential matrices,
//   H = NP + KE + sum_j w_j EP_j,
// through readPackedMatrixAccum (matrixSubs.F90:339-375), whose factor rule
// is: a factor of exactly 0.0 adds the matrix unscaled (that is how KE is
// added), any other factor multiplies it -- so a potential coefficient of
// exactly zero adds its term with weight one.  It then unpacks H and the
// overlap S into the upper triangle of full matrices (unpackMatrix,
// matrixSubs.F90:405-433) for zhegv(1, 'V', 'U').  Here both triangles are
// written (the lower as the conjugate), so any Hermitian solver can take
// them, column-major [k][col][row] as the reference's valeVale.
#include <algorithm>

#include "intg.cuh"

namespace imago {
namespace {

__global__ void k_secular(int V, long long np, int nk, int pot_dim,
                          const double *npm, const double *ke, const double *ep,
                          const double *w, const double *ol, double2 *h,
                          double2 *s) {
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

}  // namespace
}  // namespace imago

extern "C" int imago_secular_matrices(int vale_dim, int num_kpoints, int pot_dim,
                                      const double *np_packed,
                                      const double *ke_packed,
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
      vale_dim, np, num_kpoints, pot_dim, np_packed, ke_packed, ep_packed,
      pot_coeffs, ol_packed, reinterpret_cast<double2 *>(h_full),
      reinterpret_cast<double2 *>(s_full));
  if (cudaGetLastError() != cudaSuccess) return IMAGO_ERR_CUDA;
  return IMAGO_OK;
}
