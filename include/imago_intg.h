/*
 * imago_intg.h -- C ABI of the B200 integral setup for Imago.
 *
 * This library replaces the four integral builds that Imago's setupSCF
 * (src/imago/imago.F90:103-377) calls on every SCF run:
 *
 *   gaussOverlapOL      src/imago/integrals.F90:151   (called imago.F90:262)
 *   gaussOverlapKE      src/imago/integrals.F90:656   (called imago.F90:268)
 *   gaussOverlapNP      src/imago/integrals.F90:1531  (called imago.F90:284)
 *   elecPotGaussOverlap src/imago/integrals.F90:2357  (called imago.F90:293)
 *
 * and the builds beside them: gaussOverlapMV (integrals.F90:1091, rel = 1),
 * gaussOverlapHamPSCF (integrals.F90:2860), gaussOverlapDM / gaussOverlapMM
 * / gaussKOverlap (integrals3Terms.F90:64, 511, 956).  For the SCF step
 * that consumes them it provides the secular matrices (secularEqn.F90),
 * batched Hermitian eigenvalues and eigenvectors (after zhegv's Cholesky
 * reduction) and the density traces of makeValenceRho (valeCharge.F90).
 *
 * Each build sums the two- or three-centre Gaussian integrals over lattice
 * images within the reference's cutoffs, phases them onto every k-point,
 * core-orthogonalises the valence-valence block and writes it packed exactly
 * as orthoOL/ortho (integrals.F90:3608-3911, intgOrtho.F90:115-213) hand it to
 * HDF5:
 *
 *   packed[k][idx][2], idx = j*(j+1)/2 + i for 0 <= i <= j < valeDim
 *   (the Fortran column-major upper triangle, (re, im) pairs), with
 *   |x| < 1e-10 set to 0 when coreDim > 0 (intgOrtho.F90:185-190).
 *
 * The OL build also returns coreValeOL (integrals.F90:3686-3694 writes it as
 * separate real and imaginary datasets): cv_re[k][v][c], cv_im[k][v][c],
 * i.e. a column-major (coreDim, valeDim) matrix per k.
 * EP output is ordered by potential term as the reference numbers them
 * (potTypes(t)%cumulAlphaSum + alphaIndex, integrals.F90:3778):
 * ep_packed[term][k][idx][2].
 *
 * All arrays are plain FP64; all indices in the system description are the
 * reference's 1-based ones.  Every entry point returns an imago status code;
 * imago_strerror() gives the message the reference would have written to
 * fort.20 before `stop`.
 */
#ifndef IMAGO_INTG_H
#define IMAGO_INTG_H

#include <stddef.h>

#if defined(__GNUC__)
#define IMAGO_API __attribute__((visibility("default")))
#else
#define IMAGO_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  They replace the reference's `stop` statements. */
enum imago_status {
  IMAGO_OK = 0,
  IMAGO_ERR_INVALID = 1,      /* malformed system description (input.f90 checks) */
  IMAGO_ERR_CELL_LIST = 2,    /* "More lattice points needed", integrals.F90:378-383 */
  IMAGO_ERR_NEED_OVERLAP = 3, /* KE/NP/EP requested before OL while coreDim > 0 */
  IMAGO_ERR_NOMEM = 4,        /* host or device allocation failed */
  IMAGO_ERR_CUDA = 5,         /* a CUDA call failed */
  IMAGO_ERR_TIMEOUT = 6,      /* a bounded device wait gave up */
  IMAGO_ERR_NO_DEVICE = 7,    /* no CUDA device of compute capability 10.0 */
  IMAGO_ERR_RANGE = 8,        /* argument outside the supported range */
  IMAGO_ERR_SCF = 9           /* "Total energy is positive!", potentialUpdate.F90:1261-1272 */
};

/* Matrix selection bits for imago_intg_build. */
enum imago_matrix {
  IMAGO_OL = 1u, /* overlap, timeStamp 8 */
  IMAGO_KE = 2u, /* kinetic energy, timeStamp 9 */
  IMAGO_NP = 4u, /* nuclear potential, timeStamp 10 */
  IMAGO_EP = 8u, /* every electronic potential term, timeStamp 11 */
  IMAGO_MV = 16u /* mass velocity (rel = 1 only), timeStamp 30 */
};

/*
 * System description: the module data that setupSCF has read before the
 * integral calls (atomTypes, atomSites, potTypes, potSites, realVectors,
 * kPoints, logBasisFnThresh).
 */
typedef struct imago_system {
  /* realVectors(xyz, abc) in bohr, column-major: real_vectors[3*abc + xyz]
   * (lattice.f90:163, CELL_VECTORS). */
  double real_vectors[9];
  /* BASISFUNCTION_AND_ELECTROSTATIC_CUTOFFS (input.f90:327-346). */
  double basis_fn_convg;
  double electro_convg;

  /* Atom types (atomicTypes.f90:132-361). */
  int num_atom_types;
  const int *type_element;        /* elementID per type (1-based) */
  const int *type_num_orb_alphas; /* NUM_ALPHA_S_P_D_F: [4*t + l] */
  const double *type_alphas;      /* ALPHAS: numOrbAlphas(1) per type, concatenated */
  const int *type_num_core_fns;   /* radial functions per type (core) */
  const int *type_num_vale_fns;   /* radial functions per type (valence) */
  const int *fn_l;                /* QN_l per radial fn, per type core fns then
                                     valence fns, concatenated over types */
  const double *fn_coeffs;        /* numOrbAlphas(l+1) coefficients per radial
                                     fn, same order as fn_l */

  /* Atom sites (atomicSites.f90:85-132). */
  int num_atom_sites;
  const int *site_type;           /* atomTypeAssn (1-based) */
  const double *site_pos;         /* cartPos: [3*s + xyz], bohr */

  /* Potential types (potTypes.f90:86-195). */
  int num_pot_types;
  const int *pot_type_element;
  const double *pot_type_nuc_charge;
  const double *pot_type_nuc_alpha;
  const int *pot_type_num_alphas;
  const double *pot_type_alphas;  /* numAlphas per type, concatenated, ascending */

  /* Potential sites (potSites.f90:40-86): sites of one type consecutive,
   * types in ascending order. */
  int num_pot_sites;
  const int *pot_site_type;
  const double *pot_site_pos;     /* [3*s + xyz], bohr */

  /* k-points in fractional reciprocal-cell (abc) coordinates, as listed in
   * fort.15 or made by imago_kpoint_mesh (kpoints.f90:195-440). */
  int num_kpoints;
  const double *kpoints_abc;      /* [3*k + abc] */
} imago_system;

typedef struct imago_opts {
  int device;            /* CUDA device ordinal */
  void *stream;          /* cudaStream_t to run on; NULL: a private stream */
  int outputs_on_device; /* 1: output pointers are device memory */
  size_t scratch_bytes;  /* device scratch budget; 0: a quarter of free memory */
} imago_opts;

typedef struct imago_out {
  double *ol_packed; /* [nk][nPacked][2] */
  double *ol_cv_re;  /* [nk][valeDim][coreDim] */
  double *ol_cv_im;  /* [nk][valeDim][coreDim] */
  double *ke_packed; /* [nk][nPacked][2] */
  double *np_packed; /* [nk][nPacked][2] */
  double *ep_packed; /* [potDim][nk][nPacked][2] */
  double *mv_packed; /* [nk][nPacked][2], IMAGO_MV only */
} imago_out;

/* Sizes of a created context. */
typedef struct imago_dims {
  int vale_dim;      /* valeDim (atomicSites.f90:172-186) */
  int core_dim;      /* coreDim */
  int num_kpoints;
  int pot_dim;       /* potDim: sum of potential alphas over types */
  int num_cells;     /* numCellsReal (lattice.f90:310-444) */
  long long packed;  /* valeDim*(valeDim+1)/2 */
  long long num_pair_images;  /* (atom pair, lattice image) units within cutoffs */
  long long num_shell_pairs;  /* screened primitive (pair, image, alpha1, alpha2) */
  long long block_elements;   /* sum over units of n_i * n_j (states of the two
                                 atoms): the real blocks one build phases */
} imago_dims;

typedef struct imago_ctx imago_ctx;

/* Validate the system, build the lattice cell list, k-points, phase
 * factors and screening tables, and stage them on the device.  Replaces the
 * setup that setupSCF does before the integral calls
 * (imago.F90:185-258: initializeLattice, initializeFindVec,
 * initializeKPoints, renormalizeBasis, makeAlphaDist, makeAlphaNucDist,
 * makeAlphaPotDist). */
IMAGO_API int imago_intg_create(const imago_system *sys, const imago_opts *opts,
                      imago_ctx **out_ctx);

/* Fill *dims for a created context. */
IMAGO_API int imago_intg_dims(const imago_ctx *ctx, imago_dims *dims);

/* Overlap: replaces gaussOverlapOL + orthoOL (integrals.F90:151-652,
 * 3608-3745).  Must run first when coreDim > 0: the context keeps
 * coreValeOL on the device for the other builds' orthogonalisation. */
IMAGO_API int imago_gauss_overlap_ol(imago_ctx *ctx, double *packed, double *cv_re,
                           double *cv_im);

/* Kinetic energy: replaces gaussOverlapKE + ortho(2)
 * (integrals.F90:656-1090). */
IMAGO_API int imago_gauss_overlap_ke(imago_ctx *ctx, double *packed);

/* Nuclear potential: replaces gaussOverlapNP + nuclearPE + ortho(3)
 * (integrals.F90:1531-1942, 2533-2698). */
IMAGO_API int imago_gauss_overlap_np(imago_ctx *ctx, double *packed);

/* Mass velocity, the scalar-relativistic term the reference builds when
 * rel == 1: replaces gaussOverlapMV + ortho(5) (integrals.F90:1091-1527,
 * called at imago.F90:270-275).  The kinetic build's screening and lattice
 * sums with massVel2CIntg accumulated negatively.  Needs the overlap first
 * when coreDim > 0. */
IMAGO_API int imago_gauss_overlap_mv(imago_ctx *ctx, double *packed);

/* Momentum matrices, the x, y and z components of -i<a|d/dx_c|b>
 * (Hermitian): replaces gaussOverlapMM + ortho3Terms(7)
 * (integrals3Terms.F90:511-951, 1388-1608; called at imago.F90:315 and 709
 * for optical properties).  packed: [3][nk][nPacked][2].  Needs the overlap
 * first when coreDim > 0. */
IMAGO_API int imago_gauss_overlap_mm(imago_ctx *ctx, double *packed);

/* Dipole matrices, the x, y and z components of <a|(r - center)_c|b>:
 * replaces gaussOverlapDM + ortho3Terms(6) (integrals3Terms.F90:64-507;
 * called at imago.F90:312 and 705).  center is the reference's dipoleCenter
 * (input.f90:552-594), Cartesian, in bohr.  packed: [3][nk][nPacked][2]. */
IMAGO_API int imago_gauss_overlap_dm(imago_ctx *ctx, const double center[3],
                                     double *packed);

/* populateStates (populate.F90:150-620) on the host: populateStandard
 * and, when thermal_sigma is not zero, populateSmearing.  eigenvalues
 * [nk][spin][numStates] (Hartree), kpoint_weights [nk] or NULL for the mesh
 * weights 2 / nk (kpoints.f90:816); thermal_sigma, max_thermal_range and
 * fermi_search_limit as the reference holds them after input.f90:369-383
 * (sigma and limit in Hartree, the range in units of sigma).  population
 * [nk][spin][numStates] receives electronPopulation; info[5] the highest
 * occupied energy (the Fermi level when smearing), the band gap, the gap
 * kind (0 metal, 1 direct, 2 indirect), the 0-based sorted index of the
 * highest occupied state and the number of Fermi-level bisections.
 * IMAGO_ERR_RANGE when the states hold fewer than num_electrons.  No
 * device work. */
IMAGO_API int imago_populate_states(int num_kpoints, int spin, int num_states,
                                    const double *eigenvalues,
                                    const double *kpoint_weights, double num_electrons,
                                    double thermal_sigma, double max_thermal_range,
                                    double fermi_search_limit, double *population,
                                    double *info);

/* populateStates as above, also returning the sorted list the reference
 * keeps in module O_Populate (populate.F90:250-287) and frees in
 * cleanUpPopulation (populate.F90:1230-1231): sorted_energies
 * [nk * spin * numStates] receives sortedEnergyEigenValues (ascending,
 * stable) and sort_index the 0-based position of each sorted value in
 * `eigenvalues` (indexEnergyEigenValues minus 1).  Either may be NULL.
 * IMAGO_ERR_RANGE when sort_index is given and nk * spin * numStates
 * exceeds INT_MAX. */
IMAGO_API int imago_populate_states_sorted(int num_kpoints, int spin, int num_states,
                                           const double *eigenvalues,
                                           const double *kpoint_weights,
                                           double num_electrons, double thermal_sigma,
                                           double max_thermal_range,
                                           double fermi_search_limit, double *population,
                                           double *info, double *sorted_energies,
                                           int *sort_index);

/* The traces of makeValenceRho (valeCharge.F90:218-291) on the device:
 *   traces[m * nrho + s] = sum over k of matrixElementMult(M_m(k), R_s(k))
 *     = sum_k [ 2 sum_{off-diagonal} (Re M Re R + Im M Im R)
 *               + sum_{diagonal} Re M Re R ]   (matrixSubs.F90:66-109)
 * for nmat packed Hermitian matrices mats [nmat][nk][nPacked][2] (OL, NP,
 * KE, MV or the potential terms EP_j) and nrho (1 or 2) packed densities
 * rho [nrho][nk][nPacked][2] (for spin 2 the reference's total and
 * difference densities).  All pointers are device memory; the call is
 * ordered on `stream` and does not synchronise.  The partial sums are
 * added in a fixed order, so the result is reproducible. */
IMAGO_API int imago_packed_traces(int vale_dim, int num_kpoints, int nmat,
                                  const double *mats, int nrho, const double *rho,
                                  double *traces, void *stream);

/* The overlap with a plane wave, <a|exp(-i dK_c . r)|b> for three wave
 * vectors dK_c (dk[3*c .. 3*c+2], bohr^-1; the reference passes
 * recipVectors(:, c) / numAxialKPoints(c)): replaces gaussKOverlap +
 * ortho3Terms(8) (integrals3Terms.F90:956-1384, 1388-1608; called at
 * imago.F90:319 for the Berry-phase polarisation).  The matrices are not
 * Hermitian, so they are returned whole as real and imaginary planes,
 * re/im[(c * nk + k) * valeDim * valeDim + col * valeDim + row], unscreened.
 * Needs the overlap first when coreDim > 0. */
IMAGO_API int imago_gauss_koverlap(imago_ctx *ctx, const double dk[9], double *re,
                                   double *im);

/* The PSCF Hamiltonian: replaces gaussOverlapHamPSCF + orthoHamPSCF
 * (integrals.F90:2860-3606, 3913-4043; called at imago.F90:685).  One
 * matrix per spin: kinetic + nuclear + sum_t coeffs(t, q) EP_t, minus the
 * mass velocity when rel != 0, orthogonalised like KE.  coeffs is the
 * reference's potCoeffs(potDim, spin), column-major: coeffs[q * potDim + t].
 * packed: [spin][nk][nPacked][2].  spin is 1 or 2.  Needs the overlap first
 * when coreDim > 0. */
IMAGO_API int imago_ham_pscf(imago_ctx *ctx, int spin, const double *coeffs, int rel,
                             double *packed);

/* How imago_ham_pscf sums the potential terms (no counterpart in the
 * reference): 0 chooses by spin count and system size, 1 builds each
 * term's primitive blocks and adds them with their weights, 2 sums all
 * terms of a shell pair in registers (one pass per spin; several lanes per
 * shell pair on small systems), 3 as 2 with one lane per shell pair.  The
 * results agree to rounding; the choice is a matter of speed. */
IMAGO_API int imago_intg_set_ham_mode(imago_ctx *ctx, int mode);

/* Every electronic potential term: replaces elecPotGaussOverlap,
 * gaussOverlapEP, electronicPE and ortho(4) for all potDim terms
 * (integrals.F90:1946-2531, 2700-2858). */
IMAGO_API int imago_elec_pot_gauss_overlap(imago_ctx *ctx, double *packed);

/* EP terms first .. first + count - 1 only (same order and layout, `packed`
 * holding `count` matrices): the elecPotGaussOverlap loop over a sub-range
 * of its terms, for spreading the terms over several GPUs or calls.  No
 * separate counterpart in the reference. */
IMAGO_API int imago_elec_pot_gauss_overlap_range(imago_ctx *ctx, int first,
                                                 int count, double *packed);

/* All matrices selected by `which` (IMAGO_OL|IMAGO_KE|IMAGO_NP|IMAGO_EP)
 * in one call; OL runs first. */
IMAGO_API int imago_intg_build(imago_ctx *ctx, unsigned which, const imago_out *out);

/* Device time in milliseconds of the stages of the last build:
 * ms[0..3] = OL, KE, NP, EP (timeStamps.f90:45-48 labels 8-11). */
IMAGO_API int imago_intg_stage_ms(const imago_ctx *ctx, double ms[4]);

/* Device milliseconds of the last build call by kernel stage, summed over
 * matrices: ms[0] primitive integrals, ms[1] basis contraction, ms[2]
 * lattice-to-k phase sums with the scatter into the global blocks, ms[3]
 * core orthogonalisation and packing.  *launches = kernels launched. */
IMAGO_API int imago_intg_kernel_stats(const imago_ctx *ctx, double ms[4],
                                      long long *launches);

IMAGO_API void imago_intg_destroy(imago_ctx *ctx);

/* No counterpart in the reference.  The column-tile width (32, 48 or 64
 * block elements) that the tensor-core phase sum measured fastest on the
 * context's first build with more than 8 k-points, and the milliseconds of
 * that trial per width (zeros and width 64 before it has run). */
IMAGO_API int imago_intg_tuning(const imago_ctx *ctx, int *bloch_width,
                                double trial_ms[3]);

/* No counterpart in the reference: the same builds as imago_intg_build,
 * replayed from a CUDA graph.  Device outputs only (outputs_on_device), on
 * the context's own stream or a non-default one.  The first call for a
 * given `which` and output set runs an eager build (its results are
 * valid) and captures the launch sequence; later calls with the same
 * arguments replay it.  Kernel timings are not recorded for replays. */
IMAGO_API int imago_intg_build_graph(imago_ctx *ctx, unsigned which,
                                     const imago_out *out);

/*
 * Batched builds of independent cells (no counterpart in the reference):
 * one context per cell, each with its own stream and scratch (by default a
 * third of the free device memory shared out over the cells), all outputs
 * on the device.  imago_batch_build takes one imago_out per cell.  Its
 * first call for an output set runs every cell's builds concurrently on the
 * cells' streams, then captures them as one CUDA graph with a branch per
 * cell, which later calls with the same outputs replay on the batch's
 * stream (opts->stream, or a stream of its own).  Returns when all cells are
 * done.
 */
typedef struct imago_batch imago_batch;
IMAGO_API int imago_batch_create(int n, const imago_system *systems,
                                 const imago_opts *opts, imago_batch **out);
IMAGO_API int imago_batch_size(const imago_batch *batch);
IMAGO_API int imago_batch_dims(const imago_batch *batch, int cell,
                               imago_dims *dims);
IMAGO_API int imago_batch_build(imago_batch *batch, unsigned which,
                                const imago_out *outs);
/* Kernels in the captured graph (0 before the first build). */
IMAGO_API int imago_batch_launches(const imago_batch *batch, long long *launches);
IMAGO_API void imago_batch_destroy(imago_batch *batch);

/*
 * The matrices of the secular equation of one SCF step (secularEqnSCF,
 * secularEqn.F90:135-186), from device-resident packed builds: for every
 * k-point H = NP + KE + sum_j w_j EP_j accumulated in that order with the
 * reference's factor rule (readPackedMatrixAccum, matrixSubs.F90:339-375: a
 * factor of exactly 0.0 adds the matrix unscaled), and S = OL, unpacked as
 * unpackMatrix does (matrixSubs.F90:405-433) into full Hermitian matrices
 * h_full, s_full [k][col][row] of (re, im) (both triangles written).  All
 * pointers are device memory; pot_coeffs holds pot_dim factors.
 */
IMAGO_API int imago_secular_matrices(int vale_dim, int num_kpoints, int pot_dim,
                                     const double *np_packed,
                                     const double *ke_packed,
                                     const double *ep_packed,
                                     const double *pot_coeffs,
                                     const double *ol_packed, double *h_full,
                                     double *s_full, void *stream);

/* imago_secular_matrices for a scalar-relativistic run (rel == 1): the
 * mass-velocity matrix is added after KE with factor 0.0, i.e. unscaled
 * (secularEqn.F90:157-163), H = NP + KE + MV + sum_j w_j EP_j.  mv_packed
 * may be null, which is imago_secular_matrices. */
IMAGO_API int imago_secular_matrices_rel(int vale_dim, int num_kpoints, int pot_dim,
                                         const double *np_packed,
                                         const double *ke_packed,
                                         const double *mv_packed,
                                         const double *ep_packed,
                                         const double *pot_coeffs,
                                         const double *ol_packed, double *h_full,
                                         double *s_full, void *stream);

/*
 * Eigenvalues of `batch` Hermitian n x n matrices (device memory, (re, im)
 * interleaved, either storage order) into w [batch][n], ascending: by
 * default through cuSOLVER's batched Hermitian eigensolver
 * (cusolverDnXsyevBatched, loaded from the process's libcusolver.so.11),
 * else by the library's cyclic Jacobi kernel with each matrix in shared
 * memory (n up to 112); imago_hermitian_set_solver chooses.  The
 * eigenvalue step of the secular equation (zhegv after its Cholesky
 * reduction, interfaces.F90:73-120).
 */
IMAGO_API int imago_hermitian_eigvals(int n, int batch, const double *a,
                                      double *w, void *stream);

/* imago_hermitian_eigvals with the eigenvectors: a is stored row-major,
 * a[b][row][col], and vec [batch][n][n] (device, (re, im) interleaved)
 * receives vec[b][row][j], the row-th component of the unit eigenvector of
 * w[b][j] (the columns of V with A V = V diag(w)).  The batched library
 * solver synchronises the stream to check its status; the Jacobi kernel
 * accumulates its rotations and runs asynchronously.  Above n = 112
 * without the batched solver: IMAGO_ERR_RANGE.  The eigenvector step of
 * zhegv(1, 'V', 'U') after its Cholesky reduction (interfaces.F90:73-120). */
IMAGO_API int imago_hermitian_eigh(int n, int batch, const double *a, double *w,
                                   double *vec, void *stream);

/* No counterpart in the reference.  Which solver imago_hermitian_eigvals
 * and imago_hermitian_eigh use, for the whole process: 0 (the default)
 * cuSOLVER's batched solver where it loads, else the Jacobi kernel; 1 the
 * Jacobi kernel up to n = 112 (the batched solver beyond); 2 the batched
 * solver only.  Measured on one B200 for 512 matrices of n = 104: 6.1 ms
 * (values) / 7.8 ms (vectors) batched against 22.5 / 33.6 ms Jacobi. */
IMAGO_API int imago_hermitian_set_solver(int mode);
IMAGO_API int imago_hermitian_solver(int *mode);

/* The Cholesky reduction of zhegv(1, 'V', 'U') (interfaces.F90:73-120:
 * zpotrf, then zhegst) for every k-point: S = L L^H (L = U^H, zpotrf's
 * factor) and A = L^-1 H L^-H.  h_full and s_full as
 * imago_secular_matrices writes them (column-major per k-point, both
 * triangles); a [num_kpoints][n][n] receives A row-major, the layout
 * imago_hermitian_eigvals/eigh take; l_packed (may be NULL)
 * [num_kpoints][n(n+1)/2] (re, im) the factor, column by column from the
 * diagonal down (L(r, j), r >= j, at j n - j (j - 1) / 2 + r - j), for
 * imago_secular_back; info [num_kpoints] (device, may be NULL) zpotrf's
 * info per k-point: 0, or the order of the first leading minor of S that
 * is not positive definite (A of that k-point is then zero).  One
 * CTA per k-point with the factor in shared memory: n up to 128
 * (IMAGO_ERR_RANGE beyond).  a must not overlap h_full or s_full.
 * Asynchronous on `stream`. */
IMAGO_API int imago_secular_reduce(int n, int num_kpoints, const double *h_full,
                                   const double *s_full, double *a, double *l_packed,
                                   int *info, void *stream);

/* The back-transformation of zhegv(1, 'V', ...) (ztrsm with the upper
 * factor): c = L^-H y for the first num_states eigenvectors y of A, vec as
 * imago_hermitian_eigh writes it (vec[k][row][j]), l_packed from
 * imago_secular_reduce; c [num_kpoints][num_states][n] state-major
 * (c[k][j][row]), each vector normalised as zhegv's (c^H S c = 1).  n up to
 * 128 (IMAGO_ERR_RANGE beyond).  Asynchronous on `stream`. */
IMAGO_API int imago_secular_back(int n, int num_kpoints, int num_states,
                                 const double *l_packed, const double *vec, double *c,
                                 void *stream);

/* The valence density of makeValenceRho (valeCharge.F90:181-192): per
 * k-point rho = sum_j f_j c_j c_j^H over the first num_states states, the
 * zher updates in state order, packed as packMatrix leaves the upper
 * triangle ((r, q), r <= q, at q (q + 1) / 2 + r; the diagonal real).  c
 * state-major [num_kpoints][ld_states][n] (imago_secular_back's layout),
 * population [num_kpoints][ld_states] (device), rho
 * [num_kpoints][n(n+1)/2] (re, im).  Asynchronous on `stream`. */
IMAGO_API int imago_packed_density(int n, int num_kpoints, int ld_states, int num_states,
                                   const double *c, const double *population, double *rho,
                                   void *stream);

/* No counterpart: how the three-centre primitive stage of NP and EP
 * schedules its shell-pair classes.  mode 0: one launch per class
 * (k_prim3c<la, lb>), one (shell pair, term) per thread; mode 1: all
 * classes in one persistent launch whose warps take 32 items at a time
 * from a device work queue (one atomic counter), the classes ordered by
 * cost so that the cheap ones fill in behind the expensive ones; mode 2:
 * one launch per class with two EP terms of a potential type per thread
 * for the classes up to d-p (k_prim3c_pair), which walk the sites and
 * images once for both; mode -1 (the default): all run once on the
 * context's first EP build and the fastest is kept.  NP is the same bit for
 * bit under every mode, EP the same to rounding (mode 2 may enumerate an
 * item's images from another lattice vector).  A captured graph of the
 * context is dropped. */
IMAGO_API int imago_intg_set_schedule(imago_ctx *ctx, int mode);
/* The schedule in use (0, 1 or 2) and the trial times of the measurement
 * (ms, in mode order; zero when not measured). */
IMAGO_API int imago_intg_schedule(const imago_ctx *ctx, int *schedule, double trial_ms[3]);

/* No counterpart in the reference (the orthogonalisation of
 * makeValeVale/coreValeCoreCore, intgOrtho.F90:23-213, as scheduled on the
 * GPU).  For EP builds of several terms whose overlap blocks fit in shared
 * memory, mode 1 runs the persistent kernel that keeps S(k) resident and
 * brings each term's core-valence block in by TMA while the previous one
 * is reduced, mode 0 one CTA per (k, term); -1 (the default) times both on
 * the first EP build and keeps the faster.  Results are identical.  A
 * copy that does not land within its bound (1 s) makes the call return
 * IMAGO_ERR_TIMEOUT. */
IMAGO_API int imago_intg_set_ortho_schedule(imago_ctx *ctx, int mode);
/* No counterpart: the EP terms each contraction CTA handles (4 or 8),
 * measured on the context's first build of more than four terms, and the
 * trial times (ms, 4 then 8; zero when not measured). */
IMAGO_API int imago_intg_contract_tuning(const imago_ctx *ctx, int *terms_per_cta,
                                         double trial_ms[2]);
/* No counterpart in the reference.  Runs the bounded device wait that the
 * TMA-fed orthogonalisation uses on a barrier that nothing completes, with
 * a limit of limit_ms (0 < limit_ms <= 1000), on `device`'s default stream:
 * *status receives IMAGO_ERR_TIMEOUT when the wait gave up as designed and
 * the device stays usable.  Returns IMAGO_OK unless the check itself could
 * not run. */
IMAGO_API int imago_wait_check(int device, double limit_ms, int *status);

/* No counterpart in the reference.  The screened primitive triples that a
 * build evaluates -- (shell pair, potential site, lattice image) passing
 * the screens of nuclearPE (which = IMAGO_NP) or electronicPE over every
 * potential term (IMAGO_EP), integrals.F90:2533-2858 -- per shell-pair
 * class, counts[la * 4 + lb] for l = 0..3 (s, p, d, f).  Classes with f
 * are not counted (-1 where the system has them).  Synchronous on the
 * context's stream; used for the primitive stage's roofline. */
IMAGO_API int imago_intg_count_triples(imago_ctx *ctx, unsigned which, long long counts[16]);
/* The orthogonalisation schedule in use (0 or 1) and the trial times of the
 * measurement (ms, mode 0 then mode 1; zero when not measured). */
IMAGO_API int imago_intg_ortho_schedule(const imago_ctx *ctx, int *schedule,
                                        double trial_ms[2]);

/* No counterpart in the reference.  The builds of one call run each kind
 * (OL, KE, NP, EP) on a stream of its own, concurrently; serial != 0 runs
 * them one after another on the context's stream instead, which gives each
 * kernel stage its own device time in imago_intg_kernel_stats. */
IMAGO_API int imago_intg_set_serial(imago_ctx *ctx, int serial);

/* No counterpart in the reference.  Device scratch of every context comes
 * from one stream-ordered memory pool per device that keeps freed memory
 * for the next context; this hands the pool's unused memory on `device`
 * back to the driver (cudaMemPoolTrimTo). */
IMAGO_API int imago_trim_memory(int device);

IMAGO_API const char *imago_strerror(int status);

/* Monkhorst-Pack style mesh of kpoints.f90:837-899 without symmetry
 * folding (the P1 case): k_abc = -1/2 + (i - 1 + shift)/n for each axis,
 * a-major.  Writes n[0]*n[1]*n[2] points to kpoints_abc[3*k + abc]. */
IMAGO_API int imago_kpoint_mesh(const int n[3], const double shift[3],
                      double *kpoints_abc);

/*
 * Primitive integrals on the device, for checking the kernels against the
 * reference's generated primitives (gaussIntegrals.f90).  kind: 0 overlap
 * (overlap2CIntg), 1 kinetic (kinetic2CIntg), 2 three-centre overlap
 * (electron3CIntg), 3 three-centre nuclear (nuclear3CIntg), 4 Boys function
 * (boys, F_0..F_6 of params[0]), 5 mass velocity (massvel2CIntg), 6..8
 * the x, y, z components of momentum2CIntg and 9..11 those of dipole3CIntg
 * (operator centre C).  Record r reads
 *   params[r*12 + 0..11] = a1, a2, a3, A[3], B[3], C[3]
 * and cls[2*r + 0..1] = l of atom 1 and atom 2 (0..3); it writes
 * sh[r*256 + i*16 + j] = reference sh(i+1, j+1).  Host pointers.
 */
IMAGO_API int imago_prim_eval(int kind, int n, const double *params, const int *cls,
                    double *sh);

/* Records one imago_prim_eval_static call accepts, and the device memory
 * its fixed scratch array occupies on every GPU that loads this library,
 * for as long as the library stays loaded (1,101,824 bytes). */
#define IMAGO_PRIM_STATIC_MAX_RECORDS 512
#define IMAGO_PRIM_STATIC_BYTES 1101824

/*
 * imago_prim_eval without any device allocation; no counterpart in the
 * reference.  For callers that cannot call cudaMalloc: a process sharing a
 * GPU under a fixed memory budget or whose device memory already belongs to
 * a pool allocator, or a loop that cannot take the device-wide
 * synchronisation of cudaMalloc/cudaFree.  Same arguments, layout and
 * results as imago_prim_eval; the records are staged in one fixed
 * module-scope device array instead of per-call buffers.  n above
 * IMAGO_PRIM_STATIC_MAX_RECORDS returns IMAGO_ERR_RANGE.  Every call looks
 * up the array's device address on the current device
 * (cudaGetSymbolAddress, whose first use on a device loads the module and
 * should precede any stream capture there), so the address stays right
 * after a cudaDeviceReset.  Calls share the array: calls that overlap on
 * the GPU race and must not be issued.
 */
IMAGO_API int imago_prim_eval_static(int kind, int n, const double *params,
                                     const int *cls, double *sh);

#ifdef __cplusplus
}
#endif

#endif /* IMAGO_INTG_H */
