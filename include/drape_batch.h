/*
 * Batched drapes (libdrape_cuda.so): many independent garments, each on its own body, advanced together on one GPU.
 *
 * No counterpart in the reference. The reference drives one Solver per scene, and a scene with several garments
 * shares one global PCG, one line search and one convergence test (libs/sim/src/cpu_solver.cpp:169-284,
 * libs/sim/src/gpu/gpu_solver_core.cpp:312-407). A batch keeps every garment's solve separate: each garment has its
 * own Newton loop, PCG reductions, convergence test, line search, substep count and drape runner state
 * (libs/sim/src/drape_session.cpp:32-95). Only the launches are shared:
 *   - one persistent cooperative launch per Newton iteration covers every garment; each garment gets its own group
 *     of co-resident blocks, sized by its share of the work;
 *   - a frame's launches (H2D per-garment control, substeps, Newton iterations, statistics, D2H of the statistics)
 *     are one CUDA graph, replayed frame after frame;
 *   - an autotuner picks the solve kernel's lanes per block row and block size by timing them on the batch.
 *
 * Each garment is added as its own scene (drape_scene_desc with exactly one garment and its own body field). Its
 * results are those of a drape_solver built from the same scene, up to the order of floating-point reductions.
 *
 * Return codes and drape_batch_last_error() follow include/drape_cuda.h.
 */
#ifndef DRAPE_BATCH_H
#define DRAPE_BATCH_H

#include "drape_cuda.h"
#include "drape_precond.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct drape_batch drape_batch;

int drape_batch_create(int device, drape_batch** out);
void drape_batch_destroy(drape_batch* b);
const char* drape_batch_last_error(const drape_batch* b);

/* Adds one garment (a scene with garment_count == 1 and its own body; the samples are copied). Allowed until
   drape_batch_build. *index gets the garment's index in the batch. */
int drape_batch_add(drape_batch* b, const drape_scene_desc* scene, uint32_t* index);

/* Builds every garment's model, uploads the batch and partitions the launches. */
int drape_batch_build(drape_batch* b);

/* Learned preconditioner for every garment's solves (NULL: block-Jacobi), as drape_cuda_set_precond. */
int drape_batch_set_precond(drape_batch* b, drape_precond* p);

typedef struct drape_batch_tuning {
  int32_t row_lanes;      /* the PCG's product A p: 0 = slot-parallel (each thread a run of consecutive block
                             slots, row sums through shared memory), or 2, 4, 8 lanes per block row (also the lanes of
                             the learned factor's products; 4 with slot-parallel) */
  int32_t block_threads;  /* threads per block of the solve launch: 256, 512 or 1024 (1024 / this blocks per SM) */
  int32_t blocks;         /* blocks of the solve launch */
  int32_t variants_timed; /* 0 when set by hand */
  double ms_per_newton;   /* the chosen variant's mean solve time per Newton iteration during tuning */
} drape_batch_tuning;

/* Times the 12 solve variants (product scheme x block size) on the batch's current state for `frames` frames each
   (restoring the state after each) and keeps the fastest. */
int drape_batch_autotune(drape_batch* b, int frames, drape_batch_tuning* out);
/* Sets the variant by hand (row_lanes and block_threads of *tuning; the other fields are written back). */
int drape_batch_set_tuning(drape_batch* b, drape_batch_tuning* tuning);

/* One frame for every garment: max(1, substeps) substeps of dt / substeps, each with max(1, iterations) Newton
   iterations (Solver::step, solver.hpp:91, per garment). */
int drape_batch_step(drape_batch* b, double dt, int substeps, int iterations);

/* Solver::setPhase for garment `index` (entering Assembling resets its clock and re-measures its seam gaps). */
int drape_batch_set_phase(drape_batch* b, uint32_t index, int phase);

/* drapeToRest for every garment at once (DrapeSession per garment): results[i] is garment i's, `count` must equal the
   garment count; settle_seconds[i] (may be NULL) gets the wall time from the start of the call until garment i
   settled, failed or timed out. options may be NULL for the defaults. */
int drape_batch_drape_to_rest(drape_batch* b, const drape_drape_options* options, drape_drape_result* results,
                              double* settle_seconds, uint32_t count);

int drape_batch_size(const drape_batch* b, uint32_t* garments, uint64_t* particles, uint64_t* block_slots);
/* Garment `index`'s particle count and its positions (3 floats per particle). */
int drape_batch_particle_count(const drape_batch* b, uint32_t index, uint32_t* count);
int drape_batch_read_positions(const drape_batch* b, uint32_t index, float* out, size_t count);
/* Solver::stats of garment `index`, reduced on the device in FP64. */
int drape_batch_stats(drape_batch* b, uint32_t index, drape_stats* out);
/* Work counters of garment `index` since the last reset (all garments are reset together). */
int drape_batch_counters(const drape_batch* b, uint32_t index, drape_counters* out);
int drape_batch_reset_counters(drape_batch* b);

/* Snapshot of the whole batch in device memory (positions, velocities, contact state, phases, clocks, seam gaps)
   and its restore, for repeated timing from one initial state. */
int drape_batch_save(drape_batch* b);
int drape_batch_restore(drape_batch* b);

typedef struct drape_batch_profile {
  int64_t frames;            /* frames run since profiling was enabled */
  int64_t graph_launches;    /* frames replayed from the captured CUDA graph */
  int64_t solve_launches;    /* persistent solve launches (one per Newton iteration of the frame) */
  double solve_ms;           /* device time of the solve launches */
  double frame_ms;           /* device time of whole frames */
  int64_t kernel_launches;   /* kernels launched (graph nodes included) */
  int64_t cg_iterations;     /* PCG iterations summed over garments */
  double pcg_bytes;          /* algorithmic bytes of the solve launches: per PCG iteration 40 per block slot + 200
                                per particle, per FP64 energy pass 48 per stretch term + 32 per hinge + 16 per seam
                                + 96 per particle, summed over garments */
} drape_batch_profile;
/* Profiling brackets each frame and each solve launch with CUDA events (frames then run without the graph, so the
   solve launches can be timed); enabling clears the figures. */
int drape_batch_set_profiling(drape_batch* b, int enable);
int drape_batch_profile_read(const drape_batch* b, drape_batch_profile* out);

/* The batch's CUDA stream (a cudaStream_t). */
int drape_batch_stream(const drape_batch* b, void** stream);

#ifdef __cplusplus
}
#endif

#endif /* DRAPE_BATCH_H */
