/*
 * imago_learned.h -- C ABI of the learned SCF start: per-atom environment
 * descriptors and a small multilayer perceptron, trained and evaluated by
 * the library's own CUDA kernels.
 *
 * No counterpart in the reference.  Imago starts every SCF from the
 * atomic-superposition potential read by initPotCoeffs
 * (src/imago/potential.f90:433-563).  The learned start maps each atom's
 * radial environment to a correction of that start; the caller (the Python
 * host, imago_b200/learned.py) averages the corrections over the atoms of
 * each potential type, keeps the plain start as the fallback and the yardstick, and
 * discards a learned start that does not reach the plain start's energy or
 * takes more iterations.
 *
 * Descriptors: for atom i, x_k = sum over atoms j and lattice images R with
 * 0 < r = |pos_j + R - pos_i| < r_c of exp(-(r - mu_k)^2 / (2 w^2)) f_c(r),
 * f_c(r) = (cos(pi r / r_c) + 1) / 2, centres mu_k evenly spaced from
 * r_c / nrad to r_c; then a one-hot of the atom's species.
 *
 * Network: FP32 weights and FP32 accumulation, two hidden layers of tanh
 * units, a linear output: y = W3 tanh(W2 tanh(W1 x + b1) + b2) + b3.
 * Parameters are one flat FP32 array: W1 [n_in][n_hidden], b1 [n_hidden],
 * W2 [n_hidden][n_hidden], b2, W3 [n_hidden][n_out], b3 [n_out].
 * The loss is the masked mean squared error sum m (y - t)^2 / sum m.
 * Training uses Adam.  All x, t, m, y pointers are device memory (row
 * major, one row per atom); calls are ordered on the context's stream.
 */
#ifndef IMAGO_LEARNED_H
#define IMAGO_LEARNED_H

#include "imago_intg.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct imago_mlp imago_mlp;

/* A network with Xavier-uniform weights drawn from `seed`, zero biases. */
IMAGO_API int imago_mlp_create(int n_in, int n_hidden, int n_out, unsigned long long seed,
                               int device, void *stream, imago_mlp **out);
IMAGO_API void imago_mlp_destroy(imago_mlp *mlp);
/* Number of parameters. */
IMAGO_API long long imago_mlp_num_params(const imago_mlp *mlp);
/* Copy the parameters to / from host memory. */
IMAGO_API int imago_mlp_get_params(imago_mlp *mlp, float *params);
IMAGO_API int imago_mlp_set_params(imago_mlp *mlp, const float *params);
/* y [n][n_out] = network(x [n][n_in]). */
IMAGO_API int imago_mlp_forward(imago_mlp *mlp, int n, const float *x, float *y);
/* Forward and backward pass over a batch: *loss (host) receives the masked
 * MSE; the gradient stays in the context for imago_mlp_adam_step, and is
 * copied to grad (host, imago_mlp_num_params floats) when grad is not
 * NULL.  Synchronises the stream. */
IMAGO_API int imago_mlp_loss_grad(imago_mlp *mlp, int n, const float *x, const float *t,
                                  const float *mask, float *loss, float *grad);
/* One Adam update with the last gradient (bias-corrected moments). */
IMAGO_API int imago_mlp_adam_step(imago_mlp *mlp, float lr, float beta1, float beta2,
                                  float eps);

/* Descriptors of every atom of a cell, computed on the device: real_vectors
 * [3 * abc + xyz] (bohr), pos [natoms][3], species [natoms] in
 * 0..nspecies-1, cutoff r_c and width w in bohr; x (host) receives
 * [natoms][nrad + nspecies]. */
IMAGO_API int imago_descriptors(const double *real_vectors, int natoms, const double *pos,
                                const int *species, int nspecies, double cutoff, int nrad,
                                double width, int device, float *x);

#ifdef __cplusplus
}
#endif

#endif
