/*
 * lbm_closure.h -- C ABI of the learned sub-grid closure and its trainer.
 *
 * The reference has no turbulence model beyond its plain BGK collide
 * (volumetric-grid/lattice-boltzmann/shaders/collide.comp.glsl:39-61); this
 * part has no counterpart there.  It extends the physics-mode Smagorinsky
 * collide: a per-node MLP maps the node's non-equilibrium momentum flux to a
 * factor r >= 0 on the Smagorinsky constant, Cs^2 = smagorinsky_cs^2 * r,
 * evaluated inside the step kernel.  The network is trained on the GPU from
 * box-filtered fine-grid runs by the kernels below.
 *
 * Network: 9 inputs -> 32 ReLU -> 32 ReLU -> 1 softplus.  A network is an
 * array of LBM_CLOSURE_FLOATS floats:
 *   [0, 288)     W1[32][9]   (row i = hidden unit i)
 *   [288, 320)   b1[32]
 *   [320, 1344)  W2[32][32]
 *   [1344, 1376) b2[32]
 *   [1376, 1408) W3[32]
 *   [1408]       b3
 *   [1409, 1418) input mean[9]
 *   [1418, 1427) input inverse scale[9]   (x_std = (x - mean) * iscale)
 * Weights (W1, W2, W3) are used rounded to bfloat16 (round to nearest even);
 * biases, the standardisation and all arithmetic are fp32.
 *
 * Inputs of a node, from Pi = sum_i c_i c_i (f_i - feq_i) (physical units,
 * components xx yy zz xy xz yz) and rho:
 *   x[0..5] = Pi / |Pi|,  |Pi| = sqrt(Pi:Pi),
 *   x[6]    = log |Pi|,
 *   x[7]    = tr((Pi/|Pi|)^3),
 *   x[8]    = rho - 1.
 *
 * Device pointers are marked d_; `stream` is a cudaStream_t (NULL = the
 * legacy default stream).  Status codes as in lbm.h.
 */
#ifndef LBM_B200_CLOSURE_H
#define LBM_B200_CLOSURE_H

#include "lbm.h"

#ifdef __cplusplus
extern "C" {
#endif

#define LBM_CLOSURE_INPUTS 9
#define LBM_CLOSURE_HIDDEN 32
#define LBM_CLOSURE_PARAMS 1409
#define LBM_CLOSURE_FLOATS 1427

/* Installs a network on a physics-mode lattice whose descriptor has
 * smagorinsky_cs > 0 (the Cs0 that r scales); later steps use it.  net = NULL
 * removes it (plain Smagorinsky again).  The weights are copied.  By default
 * the step evaluates the MLP on CUDA cores (fp32 activations, the weights as
 * constant-bank operands, one or two nodes per thread);
 * lbm_set_step_variant(ctx, 8) evaluates the 32 x 32 hidden layer on the
 * tensor cores instead (tcgen05 MMA of the CTA's 128 nodes, bf16 activations
 * and weights, fp32 accumulator in tensor memory). */
LBM_API int lbm_set_closure(lbm_ctx* ctx, const float* net);

/* Testing hook of the tensor-core closure step (variant 8): the bound, in
 * polls of mbarrier.try_wait (each of which the hardware may suspend for a
 * while), of each wait for the CTA's MMAs; polls < 0 restores the default
 * (2^22), 0 makes every such wait give up at once.  A wait that runs out
 * makes that CTA issue no further MMA in the launch: its nodes fall back to
 * r = 1 (plain Smagorinsky) and lbm_sync reports LBM_ERR_TIMEOUT.  The wait
 * that keeps a CTA from freeing its tensor memory under an MMA still in
 * flight keeps the default bound, so 0 exercises the give-up path without a
 * fault.  Takes effect at the next step; the context stays usable. */
LBM_API int lbm_set_closure_wait_limit(lbm_ctx* ctx, int32_t polls);

/* Box filter of moment fields by `factor` along each axis (factor divides
 * nx, ny, nz).  d_rho float[n], d_u float[3][n] planes (as from
 * lbm_device_moments); d_out float[10][nc] planes, nc = n / factor^3, in the
 * coarse grid's x-fastest order: rho_bar (box mean of rho), the Favre
 * velocity u~ = <rho u> / <rho> (3), and the sub-filter stress
 * tau_ab = <rho u_a u_b> / <rho> - u~_a u~_b (xx yy zz xy xz yz).
 * Sums in fp64. */
LBM_API int lbm_box_filter(const float* d_rho, const float* d_u, int32_t nx, int32_t ny,
                           int32_t nz, int32_t factor, float* d_out, void* stream);

/* Training samples from a filtered field (d_filt as written by
 * lbm_box_filter, periodic grid nx*ny*nz).  Sample i takes node
 * hash(seed, i) mod n (seed 0: node i, i < n).  With the strain rate S of u~
 * by central differences and |S| = sqrt(2 S:S):
 *   target r* = -tau^d : S / (cs0^2 |S|^3)   (the Cs^2 ratio whose eddy
 *               viscosity cs0^2 r* |S| reproduces the node's sub-filter
 *               energy flux -tau:S),
 *   weight    = |S|^3,
 *   inputs    = the features of Pi = -(2/3) rho_bar tau_s S with
 *               tau_s = tau + 3 cs0^2 |S| (the flux a Smagorinsky-closed
 *               coarse node carries at that strain).
 * d_x float[n_samples][9], d_target and d_weight float[n_samples]. */
LBM_API int lbm_closure_samples(const float* d_filt, int32_t nx, int32_t ny, int32_t nz,
                                float tau, float cs0, uint64_t seed, int64_t n_samples,
                                float* d_x, float* d_target, float* d_weight, void* stream);

/* Network output r for each of n samples (d_x float[n][9] -> d_r float[n]). */
LBM_API int lbm_closure_predict(const float* net, const float* d_x, int64_t n, float* d_r,
                                void* stream);

/* ---- trainer ------------------------------------------------------------ */
typedef struct lbm_trainer lbm_trainer;

typedef struct lbm_adam {
    uint32_t struct_size;
    float    lr;            /* default 1e-3  */
    float    beta1;         /* default 0.9   */
    float    beta2;         /* default 0.999 */
    float    eps;           /* default 1e-8  */
    float    weight_decay;  /* decoupled, on W1 W2 W3; default 0 */
} lbm_adam;

LBM_API int lbm_adam_default(lbm_adam* a);
/* Owns fp32 master parameters (initialised from net), Adam moments and the
 * gradient buffers on the current device.  The input mean / inverse scale of
 * net are kept fixed. */
LBM_API int lbm_trainer_create(const float* net, const lbm_adam* opt, lbm_trainer** out);
LBM_API int lbm_trainer_destroy(lbm_trainer* t);
LBM_API int lbm_trainer_set_stream(lbm_trainer* t, void* stream);
/* Loss L = wscale * sum_i w_i (r(x_i) - target_i)^2 over the n samples in
 * order, and its gradient with respect to the parameters (the bf16-rounded
 * weights the forward pass uses), by the fused forward/backward kernel.
 * grad: host float[LBM_CLOSURE_PARAMS] or NULL; loss: host or NULL.  The
 * gradient stays in the trainer for lbm_trainer_adam_step. */
LBM_API int lbm_trainer_grad(lbm_trainer* t, const float* d_x, const float* d_target,
                             const float* d_weight, int64_t n, float wscale, float* grad,
                             double* loss);
/* One Adam update of the master parameters from the last gradient. */
LBM_API int lbm_trainer_adam_step(lbm_trainer* t);
/* Minibatch training: `epochs` passes over the n samples in an order drawn
 * from seed (an affine permutation per epoch), batches of `batch`, each
 * loss normalised by the dataset's mean weight: L = sum_b w (r - t)^2 /
 * (batch * mean w).  epoch_loss: host double[epochs] (mean batch loss) or
 * NULL. */
LBM_API int lbm_trainer_fit(lbm_trainer* t, const float* d_x, const float* d_target,
                            const float* d_weight, int64_t n, int32_t batch, int32_t epochs,
                            uint64_t seed, double* epoch_loss);
/* Current network (bf16-rounded weights, fp32 biases, the fixed
 * standardisation): host float[LBM_CLOSURE_FLOATS]. */
LBM_API int lbm_trainer_get_net(lbm_trainer* t, float* net);
LBM_API const char* lbm_trainer_last_error(lbm_trainer* t);

/* bfloat16 rounding (nearest even) of n floats, as the kernels apply it to
 * the weights; host only. */
LBM_API int lbm_round_bf16(const float* in, float* out, size_t n);

#ifdef __cplusplus
}
#endif
#endif /* LBM_B200_CLOSURE_H */
