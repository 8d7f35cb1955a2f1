/*
 * mpmw_mlp.h -- C ABI of the learned return-map surrogate in libmpmw.so.
 *
 * No counterpart in the reference.  MPMWarpYDW's Drucker-Prager return map
 * (utils/mpmRoutines.py:314-453) is closed form; this is an optional surrogate
 * for the return of plastic trial states, with the plain map as the fallback.
 *
 * Network: 8 -> 64 -> 64 -> 64 -> 4, SiLU after each hidden layer.  Parameters
 * are one FP32 array of MPMW_MLP_NPARAM floats in this order (row-major,
 * W[out][in]): W1[64][8] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[4][64] b4[4].
 *
 * Features of a plastic trial state with principal log strains e (sorted
 * descending), in units of the yield strain y = ys / (2 mu):
 *   x = ( e/|e| (3), log10(|e| / y), alpha, beta, ln(1 - D), nu )
 * Targets, relative to the radial return's own scales (so that an output error
 * is a relative error of the returned quantity, whatever |e| / y is): with
 * n = |dev e| and rho = yield / (2 mu n) (returned over trial deviatoric norm,
 * 0 < rho < 1 for a plastic trial; yield = (1 - D)(ys - alpha p)),
 *   y = ( ln rho, ln(1 - rho),
 *         volumetric strain added to each principal component per unit
 *         plastic multiplier (beta),
 *         accumulated-plastic-strain increment per unit plastic multiplier
 *         (sqrt(2/3)) ).
 * The return follows as dgamma = n (1 - rho) + 1e-6,
 *   e_ret = e + (rho n / (n + 1e-6) - 1) dev e + y[2] dgamma,
 *   d_acc = y[3] dgamma
 * (the reference's 1e-6 offset of |dev e|, utils/mpmRoutines.py:407, is
 * applied exactly, outside the network).
 *
 * Precision: the hidden layers' weights are BF16 (training rounds them the
 * same way, straight-through); the last layer's weights and every bias are
 * FP32.  The tensor-core inference feeds each hidden-layer input to the MMAs
 * as two BF16 terms (hi + lo), so activations carry about 2^-17 relative
 * rounding; the last layer runs in FP32 on the CUDA cores.
 *
 * Conventions as in mpmw.h: device pointers, int status, stream-ordered, no
 * allocation (callers pass scratch).
 */
#ifndef MPMW_MLP_H
#define MPMW_MLP_H

#include "mpmw.h"

#ifdef __cplusplus
extern "C" {
#endif

#define MPMW_MLP_IN 8
#define MPMW_MLP_HID 64
#define MPMW_MLP_OUT 4
#define MPMW_MLP_NPARAM 9156
/* bytes of the packed BF16 weights for the tensor-core inference kernel */
#define MPMW_MLP_PACKED_BYTES 20480

/* Training set: n labelled plastic trial states drawn as
 *   |e| log-uniform in [1e-6, 1e-1], direction uniform on the sphere,
 *   friction angle U(20, 45) deg -> alpha; beta = 0.3 alpha (the reference's
 *   dilation, utils/mpmRoutines.py:424) for half the samples, else a dilation
 *   angle U(0, 10) deg -> beta;
 *   cohesion log-uniform in [0.1, 5] MPa, E log-uniform in [1, 50] GPa,
 *   nu U(0.15, 0.35), D U(0, MPMW_SURR_D_MAX),
 * keeping only states whose trial is plastic; labels from the plain
 * principal-space return map in double precision.  x: [n][8], y: [n][4]. */
#define MPMW_SURR_D_MAX 0.999f /* trials with more damage take the exact return */
int mpmw_dp_samples(int64_t n, uint64_t seed, float *x, float *y, mpmw_stream_t stream);

/* FP32 forward pass with the hidden layers' weights rounded to BF16 (the last
 * layer's weights and the biases FP32): y = f(x). */
int mpmw_mlp_forward(const float *params, const float *x, int64_t n, float *y, mpmw_stream_t stream);

/* Mean-squared-error loss over n samples and its gradient with respect to the
 * FP32 parameters (straight-through through the BF16 rounding of the
 * weights).  grad[MPMW_MLP_NPARAM] and loss[1] are overwritten. */
int mpmw_mlp_grad(const float *params, const float *x, const float *y, int64_t n, float *grad, float *loss,
                  mpmw_stream_t stream);

/* The same loss and gradient on the tensor cores (tcgen05.mma, FP32
 * accumulators in tensor memory), 128 samples per CTA: the forward pass as
 * mpmw_mlp_infer_tc; the back-propagated errors dz W with dz as hi + lo BF16
 * terms against the BF16 weights; the weight and bias gradients dz^T a with
 * the samples as the MMA's K (dz^T as hi + lo terms, a in BF16, a row of ones
 * for the bias); the last layer in FP32 on the CUDA cores.  Pre-activations
 * are recomputed by each layer's MMA instead of being stored.  Bounded waits
 * report MPMW_ST_TIMEOUT in *status (may be NULL). */
int mpmw_mlp_grad_tc(const float *params, const float *x, const float *y, int64_t n, float *grad, float *loss,
                     uint32_t *status, mpmw_stream_t stream);

/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8), step counts from 1. */
int mpmw_mlp_adam(float *params, const float *grad, float *m, float *v, int step, float lr, mpmw_stream_t stream);

/* Pack the FP32 weights as BF16 operand tiles for mpmw_mlp_infer_tc. */
int mpmw_mlp_pack(const float *params, void *packed, mpmw_stream_t stream);

/* Tensor-core inference (tcgen05.mma with BF16 operands, each hidden-layer
 * input split into hi + lo BF16 terms, FP32 accumulators in tensor memory;
 * the last layer in FP32 on the CUDA cores): y[n][4] = f(x[n][8]) with the
 * packed weights and the FP32 biases and last-layer weights of `params`.
 * Bounded waits report MPMW_ST_TIMEOUT in *status. */
int mpmw_mlp_infer_tc(const void *packed, const float *params, const float *x, int64_t n, float *y,
                      uint32_t *status, mpmw_stream_t stream);

/* Workspace bytes of mpmw_stress_surrogate for n particles. */
size_t mpmw_surrogate_workspace_bytes(int64_t n);

/* The stress phase (utils/mpmRoutines.py:229-312) with the surrogate for the
 * return of plastic trial states.  Particles outside the tensor form's range,
 * elastic trials and trials that set D = 1 are computed exactly as mpmw_stress
 * (MPMW_STRESS_AUTO).  A surrogate return is accepted only if it agrees with
 * the state the return's identities define (the yield condition fixes the
 * returned deviatoric norm, the flow rule the volumetric part and the
 * accumulated-strain increment): principal stresses within gate_tol
 * (relative, norm-wise) and the increment within gate_tol of the larger of
 * itself and the yield strain; otherwise the exact closed form is used.
 * audit_per_mille of the surrogate's returns (chosen by a hash of the particle
 * index and audit_seed; audited before the gate) are compared with the exact
 * return.  Trials with D > MPMW_SURR_D_MAX take the exact return.
 * stats (device, MPMW_SURR_NSTATS x uint32, accumulated; the caller zeroes
 * it): surrogate candidates, gate fallbacks, audited, largest audited relative
 * stress error (float bits), sum of audited relative errors (float bits),
 * audited within 1e-3, audited and accepted by the gate, largest audited
 * relative stress error among those accepted (float bits). */
#define MPMW_SURR_NSTATS 8
int mpmw_stress_surrogate(const mpmw_particles_t *p, const mpmw_params_t *prm, const void *packed,
                          const float *mlp_params, float gate_tol, int audit_per_mille, uint64_t audit_seed,
                          uint32_t *stats, uint32_t *status, void *workspace, size_t ws_bytes, mpmw_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* MPMW_MLP_H */
