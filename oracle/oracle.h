/*
 * oracle.h -- CPU restatement of the reference's integral setup.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * it.  Nothing in imago_b200/ links or calls it.
 *
 * Parity status: the primitive integrals and the Boys function are pinned to
 * the reference's own generated kernels (src/imago/gaussIntegrals.f90),
 * executed statement by statement to make tests/golden/primitives.json.  The
 * driver loops (lattice, screening, lattice sums, Bloch phases, saving,
 * core orthogonalisation, packing) restate src/imago/integrals.F90,
 * intgSaving.F90, intgOrtho.F90, lattice.f90, kpoints.f90, basis.f90 and
 * gaussRelations.f90 line for line; the reference is Fortran with no
 * compiler available here and ships no golden matrices, so at the driver
 * level parity is unpinned and rests on this restatement plus analytic
 * known-answer checks.
 */
#ifndef IMAGO_ORACLE_H
#define IMAGO_ORACLE_H

#include "../include/imago_intg.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Primitives: sh[i*16 + j] = reference sh(i+1, j+1); la, lb in 0..3. */
void orc_boys(double T, double F[7]);
void orc_overlap2c(double a1, double a2, const double *A, const double *B,
                   int la, int lb, double *sh);
void orc_kinetic2c(double a1, double a2, const double *A, const double *B,
                   int la, int lb, double *sh);
void orc_massvel2c(double a1, double a2, const double *A, const double *B,
                   int la, int lb, double *sh);
/* Three components: sh3[c*256 + i*16 + j] = reference sh(i+1, j+1, c+1). */
void orc_momentum2c(double a1, double a2, const double *A, const double *B,
                    int la, int lb, double *sh3);
void orc_dipole2c(double a1, double a2, const double *A, const double *B,
                  const double *C, int la, int lb, double *sh3);
/* <a|exp(-i dK.r)|b>: sh2[2*(i*16 + j) + 0/1] = Re/Im sh(i+1, j+1). */
void orc_koverlap2c(double a1, double a2, const double *A, const double *B,
                    const double *dK, int la, int lb, double *sh2);
void orc_electron3c(double a1, double a2, double a3, const double *A,
                    const double *B, const double *C, int la, int lb,
                    double *sh);
void orc_nuclear3c(double a1, double a2, double a3, const double *A,
                   const double *B, const double *C, int la, int lb,
                   double *sh);

typedef struct orc_ctx orc_ctx;

int orc_create(const imago_system *sys, orc_ctx **out);
void orc_destroy(orc_ctx *c);
int orc_dims(const orc_ctx *c, imago_dims *d);

/* Work restriction for bounded CPU samples: only atom pairs whose linear
 * index (i-major over i <= j) is a multiple of `stride` are integrated.
 * stride 1 (the default) is the full build.  nthreads <= 0: all cores. */
void orc_set_sampling(orc_ctx *c, int stride, int nthreads);
/* Timing samples only: skip the orthogonalisation and packing. */
void orc_set_skip_ortho(orc_ctx *c, int skip);

int orc_gauss_overlap_ol(orc_ctx *c, double *packed, double *cv_re,
                         double *cv_im);
int orc_gauss_overlap_ke(orc_ctx *c, double *packed);
int orc_gauss_overlap_np(orc_ctx *c, double *packed);
/* Mass velocity (rel = 1 runs only). */
int orc_gauss_overlap_mv(orc_ctx *c, double *packed);
/* Momentum (-i d/dx_c, Hermitian) and dipole (r - center)_c matrices,
 * packed [3][nk][np][2] for c = x, y, z. */
int orc_gauss_overlap_mm(orc_ctx *c, double *packed);
int orc_gauss_overlap_dm(orc_ctx *c, const double center[3], double *packed);
/* K-overlap: dk[3 * axis + xyz] the three wave vectors; re, im full
 * [3][nk][V][V] planes, column-major per k. */
int orc_gauss_koverlap(orc_ctx *c, const double *dk, double *re, double *im);
/* The PSCF Hamiltonian: packed [spin][nk][np][2]; coeffs the reference's
 * potCoeffs(potDim, spin), column-major: coeffs[q * potDim + t]. */
int orc_ham_pscf(orc_ctx *c, int spin, const double *coeffs, int rel,
                 double *packed);
/* Terms [term_lo, term_hi) of the potDim electronic potential terms;
 * packed holds (term_hi - term_lo) matrices. */
int orc_elec_pot_gauss_overlap(orc_ctx *c, int term_lo, int term_hi,
                               double *packed);

/* Seconds spent in the pair/lattice loops and in orthogonalisation by the
 * last build call. */
void orc_last_times(const orc_ctx *c, double *loops_s, double *ortho_s);

/* Lattice and k-point introspection for tests. */
int orc_num_cells(const orc_ctx *c);
void orc_cells(const orc_ctx *c, double *dims /* [n*3] */, double *sizes);
void orc_kpoints_xyz(const orc_ctx *c, double *k /* [nk*3] */);
void orc_find_lattice_vector(const orc_ctx *c, const double *v, double *out);
/* Counts of screened work units of the last build call. */
void orc_last_counts(const orc_ctx *c, long long *pair_images,
                     long long *shell_pairs, long long *triples);

#ifdef __cplusplus
}
#endif

#endif
