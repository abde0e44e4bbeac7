/* Learned preconditioner for the cloth solver's PCG: a message-passing network (4 layers, hidden 64, BF16 weights,
   FP32 accumulation on tcgen05 tensor cores) over the block-CSR graph of a Newton system, emitting a block
   lower-triangular factor L with M^-1 = L L^T. L = S G with S = blockdiag(chol(inv(A_ii))), so G = I reproduces
   block-Jacobi exactly; L's diagonal blocks are lower-triangular with a positive diagonal, so M^-1 is SPD on the
   unpinned unknowns for any weights.

   No counterpart in the reference, whose PCG is block-Jacobi only (libs/sim/src/cpu_solver.cpp:169-213,
   libs/sim/kernels/kernels.h:237-249). Status codes are those of drape_cuda.h. */
#ifndef DRAPE_PRECOND_H
#define DRAPE_PRECOND_H

#include <stddef.h>
#include <stdint.h>

#include "drape_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct drape_precond drape_precond;

/* Number of FP32 parameters; layout: [out][in] row-major weights then the bias, in the order W_ne b_ne (node encoder,
   64 x 16), W_ee b_ee (slot encoder, 64 x 16), per layer W_m b_m W_u b_u (64 x 128 each), W_o b_o (16 x 192). */
uint32_t drape_precond_param_count(void);

int drape_precond_create(int device, drape_precond** out);
void drape_precond_destroy(drape_precond* p);
/* Message of the last failed call on this handle (NULL: of the last failed create on this thread). */
const char* drape_precond_last_error(drape_precond* p);

/* FP32 master parameters (count = drape_precond_param_count()); setting them resets the optimiser state. */
int drape_precond_set_params(drape_precond* p, const float* params, size_t count);
int drape_precond_get_params(drape_precond* p, float* params, size_t count);

/* A training sample: a Newton system in host memory (CSR with sorted columns and a diagonal block in every row,
   blocks row-major 9 floats per slot, symmetric pattern), pinned and contact-active flags per particle, and
   `residual_count` residual vectors (3 n floats each). Returns the sample index in *sample. */
int drape_precond_add_sample(drape_precond* p, uint32_t n, const uint32_t* row_start, const uint32_t* col_index,
                             const float* blocks, const uint8_t* pinned, const uint8_t* active,
                             const float* residuals, uint32_t residual_count, int* sample);
int drape_precond_clear_samples(drape_precond* p);

/* Network forward on a sample: G and L = S G per slot (9 floats each, row-major; zero off the lower live slots). */
int drape_precond_forward(drape_precond* p, int sample, float* g_blocks, float* l_blocks);
/* The same network on a sample through the inference path the solver runs (slot and node GEMMs on contiguous tiles,
   message sums and the output layer as row gathers): L per slot as in drape_precond_forward, equal to it up to FP32
   summation order and one more BF16 rounding. */
int drape_precond_forward_inference(drape_precond* p, int sample, float* l_blocks);
/* Evaluation PCG on a sample (no contact filter): solves S^T A S x = S^T r, r the sample's residual `rhs`, with the
   preconditioner G G^T (use_learned != 0) or the identity, which on the scaled system is block-Jacobi; stops at
   |r_k| <= tolerance |r_0| or max_iterations. Gives both preconditioners the same system for an ablation. */
int drape_precond_pcg(drape_precond* p, int sample, int rhs, int use_learned, int max_iterations, double tolerance,
                      int* iterations, double* relative_residual);

/* Training objectives. DRAPE_PRECOND_KAPORIN (the default): log(w^T G^T Ahat G w / N) - (2 / N) log det G on a
   probe w (the sample's residual vectors, which should then be random with identity covariance), N the live
   unknowns: a stochastic estimate of Kaporin's condition number of the preconditioned operator, minimised on a fixed
   pattern by the factorised sparse approximate inverse. DRAPE_PRECOND_DEFECT: |Ahat G G^T rhat - rhat|^2 / |rhat|^2
   with rhat = S^T r. Ahat = S^T A S. */
#define DRAPE_PRECOND_DEFECT 0
#define DRAPE_PRECOND_KAPORIN 1
int drape_precond_set_objective(drape_precond* p, int objective);

/* The objective on one residual (probe) and its gradient with respect to the parameters (param_count floats; may be
   NULL). */
int drape_precond_loss_grad(drape_precond* p, int sample, int residual, double* loss, float* grad);
/* z = L L^T r on a sample (3 n floats each). */
int drape_precond_apply(drape_precond* p, int sample, const float* r, float* z);
/* `steps` Adam steps (beta 0.9 / 0.999), each on the summed gradient of `batch` (sample, residual) pairs drawn with
   the seed; losses[step] (may be NULL) gets the batch's mean loss before the step. */
int drape_precond_train(drape_precond* p, int steps, float learning_rate, int batch, uint64_t seed, float* losses);

/* Makes the solver's Newton solves use the learned preconditioner with the parameters `p` holds now (copied; `p` may
   be destroyed afterwards), or block-Jacobi again when `p` is NULL. Each Newton iteration then runs the network on
   the assembled system and the PCG applies z = F L L^T F r; a solve that breaks down (a non-finite scalar, or |r|^2
   above 1e6 |r0|^2) is restarted with block-Jacobi and counted in
   drape_counters.precond_fallbacks. The convergence test stays the reference's (cpu_solver.cpp:205-207). */
int drape_cuda_set_precond(drape_solver* s, drape_precond* p);
/* Inspection: the factor L (9 floats per slot, row-major; zero off the lower slots) of the solver's last network
   run. */
int drape_cuda_precond_factor(drape_solver* s, float* l_blocks);

/* Schedule of the learned preconditioner. The network runs on every `refresh_every`-th Newton iteration only (default
   1; the factor in between is the last one: any factor keeps M^-1 SPD, so a stale one only changes the iteration
   count; the count restarts at each build). Each PCG solve first runs `jacobi_first` block-Jacobi iterations (default
   0) and, when those have not met the convergence test, continues from the current iterate with the learned
   preconditioner within the same iteration cap: a Newton system whose right-hand side is local converges under
   block-Jacobi in a few iterations, where the learned factor's coupling to neighbours costs iterations. */
int drape_cuda_set_precond_schedule(drape_solver* s, int refresh_every, int jacobi_first);

#ifdef __cplusplus
}
#endif

#endif
