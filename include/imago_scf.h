/*
 * imago_scf.h -- C ABI of the SCF potential update on the B200.
 *
 * The SCF loop of Imago (mainSCF, src/imago/imago.F90:420-540) repeats
 * secularEqnSCF -> populateStates -> makeValenceRho -> makeSCFPot until the
 * potential converges.  imago_intg.h covers the integrals, the secular
 * matrices, the populations and the density traces; this header covers the
 * rest:
 *
 *   imago_scf_create       the SCF set-up that setupSCF does after the
 *                          integrals (imago.F90:185-377): the real and
 *                          reciprocal lattice lists (initializeLattice,
 *                          lattice.f90:310-444), the exchange-correlation
 *                          mesh and overlap (getECMeshParameters,
 *                          makeECMeshAndOverlap, exchCorr.f90:63-873), the
 *                          core charge fit (makeCoreRho, coreCharge.f90:27-578),
 *                          the electrostatic operators (makeElectrostatics,
 *                          elecStat.f90:36-1042) and the integration
 *                          constants (initPotStructures, potential.f90:109-160)
 *   imago_scf_pot_update   makeSCFPot (potentialUpdate.F90:53-1866): the charge
 *                          fit, the electrostatic and exchange-correlation
 *                          potentials and energies, the Anderson mixing of
 *                          the next potential coefficients and the
 *                          convergence test
 *
 * Scope: spin 1, rel 0, the local-density functionals XC_CODE 100 (Wigner),
 * 101 (Ceperley-Alder) and 102 (Hedin-Lundqvist), no +UJ.  Other codes
 * return IMAGO_ERR_RANGE.
 *
 * Layouts follow the reference's arrays: potential terms are numbered as
 * potTypes(t)%cumulAlphaSum + alphaIndex; potDim x potDim matrices are
 * column-major (element (r, c) at [c * potDim + r]); the mesh operator
 * exchRhoOp(term, point) is stored point by point, [point * potDim + term],
 * the points of the potential sites one after another.
 */
#ifndef IMAGO_SCF_H
#define IMAGO_SCF_H

#include "imago_intg.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct imago_scf imago_scf;

/* The SCF control input (MAIN_INPUT_DATA, input.f90 / potential.f90:344-431)
 * and the exchange-correlation mesh parameters (exchCorr.f90:876-913). */
typedef struct imago_scf_params {
  int xc_code;               /* XC_CODE */
  int feedback_level;        /* FEEDBACK_LEVEL (Anderson order 0, 1 or 2) */
  double relax_factor;       /* RELAXATION_FACTOR */
  double convergence_test;   /* CONVERGENCE_TEST */
  int num_sample_vectors;    /* NUM_ANGULAR_SAMPLE_VECTORS */
  double ang_weights[2];     /* WTIN_WTOUT */
  double r_sample[3];        /* RADIAL_SAMPLE-IN_OUT_SPACING: in, out, spacing */
  double num_electrons;      /* NUM_ELECTRONS */
  const double *covalent_radius; /* COVALENT_RADIUS per potential type, as the
                                    pot deck gives it (potTypes.f90:86-160) */
} imago_scf_params;

typedef struct imago_scf_dims {
  int pot_dim;
  int num_pot_types;
  int num_pot_sites;
  int num_cells_real;    /* numCellsReal */
  int num_cells_recip;   /* numCellsRecip */
  int num_mesh_points;   /* sum over potential sites of numRayPoints */
} imago_scf_dims;

/* Build the SCF set-up on `device` (NULL stream: a private one).  The
 * system is the one the integrals were built for (its potential types,
 * sites, atom types and cell; k-points are not used). */
IMAGO_API int imago_scf_create(const imago_system *sys, const imago_scf_params *params,
                               int device, void *stream, imago_scf **out);
IMAGO_API void imago_scf_destroy(imago_scf *scf);
IMAGO_API int imago_scf_get_dims(const imago_scf *scf, imago_scf_dims *dims);

/* The set-up results as setupSCF stores them (hdf5SCFElecStat /
 * hdf5SCFExchCorr datasets); each pointer may be NULL.  potDim x potDim
 * matrices: pot_alpha_overlap, nonlocal_neut_q, local_neut_q, xc_overlap
 * (upper triangle, as makeECMeshAndOverlap fills it); potDim vectors:
 * nonlocal_nuc_q, local_nuc_q, core_charge (coreChargeDensity), intg_consts;
 * nonlocal_residual_q [potDim][numPotTypes] (column-major
 * (numPotTypes, potDim)). */
IMAGO_API int imago_scf_setup_arrays(const imago_scf *scf, double *pot_alpha_overlap,
                                     double *nonlocal_neut_q, double *local_neut_q,
                                     double *nonlocal_nuc_q, double *local_nuc_q,
                                     double *nonlocal_residual_q, double *core_charge,
                                     double *xc_overlap, double *intg_consts);

/* The exchange-correlation mesh: site_points [numPotSites] (numRayPoints,
 * 0 for a site whose covalent radius is below smallThresh), radial_weight
 * [num_mesh_points], exch_rho_op [num_mesh_points][potDim]. */
IMAGO_API int imago_scf_mesh(const imago_scf *scf, int *site_points, double *radial_weight,
                             double *exch_rho_op);

/* The lattice lists: real_dims [numCellsReal][3], real_sizes [numCellsReal]
 * (|R|^2), recip_dims [numCellsRecip][3], recip_sizes; each may be NULL. */
IMAGO_API int imago_scf_lattice(const imago_scf *scf, double *real_dims, double *real_sizes,
                                double *recip_dims, double *recip_sizes);

/* makeSCFPot for one iteration.  pot_rho [potDim] and the three traces are
 * makeValenceRho's (potRho(:,1), chargeDensityTrace(1) is not needed,
 * nucPotTrace(1), kineticEnergyTrace(1)); pot_coeffs [potDim] holds the
 * coefficients used in this iteration and receives the next ones.
 * result[8]: total energy, kinetic energy, electrostatic energy,
 * exchange-correlation energy (Hartree), the unconstrained valence fit
 * error (electronDiff), testableDelta, converged (1/0) and the iteration
 * number after the call (currIteration).  The Anderson history of the
 * earlier calls lives in the context; imago_scf_reset_history starts a new
 * sequence at iteration 1.  IMAGO_ERR_SCF when the total energy comes out
 * positive (the reference stops there).  Synchronises the context's
 * stream. */
IMAGO_API int imago_scf_pot_update(imago_scf *scf, const double *pot_rho,
                                   double nuc_pot_trace, double kinetic_trace,
                                   double *pot_coeffs, double *result);
IMAGO_API int imago_scf_reset_history(imago_scf *scf);

/* Device time of the last imago_scf_create's electrostatics and mesh
 * kernels, and of the last update's mesh kernels, in milliseconds:
 * ms[0] electrostatics, ms[1] mesh operator and overlap, ms[2] update. */
IMAGO_API int imago_scf_timings(const imago_scf *scf, double ms[3]);

#ifdef __cplusplus
}
#endif

#endif
