/*
 * C ABI of the B200 cloth-solver hot path (libdrape_cuda.so).
 *
 * One opaque handle is one solver: the reference's drape::sim::Solver (libs/sim/include/drape/sim/solver.hpp:85-98)
 * with its state on one GPU. A reference-side CudaSolver forwards each Solver method to the
 * entry point named beside it, and registers itself as a SolverBackend in makeSolver / isAvailable / backendName
 * (libs/sim/include/drape/sim/solver_factory.hpp:12-20, libs/sim/src/solver_factory.cpp:16-61), so the GPU/CPU switch
 * (libs/session/include/drape/session/sim_controller.hpp:25) can select it.
 *
 * Every call returns an int status. The wrapper maps them to the reference's exception types:
 *   DRAPE_OK              0
 *   DRAPE_INVALID        -1  std::invalid_argument  (inconsistent scene, size mismatch: sim_model.cpp:81-86,
 *                                                   cpu_solver.cpp:340-343, sim_model.cpp:342-344)
 *   DRAPE_OUT_OF_RANGE   -2  std::out_of_range      (unknown garment id, pin/force particle out of range:
 *                                                   solver.hpp:96, sim_model.cpp:184, :190)
 *   DRAPE_DEVICE_ERROR   -3  std::runtime_error     ("cuda: <cause>", the backend-prefixed device failure of
 *                                                   metal_device.cpp:136 / solver_factory.cpp:57)
 *   DRAPE_NOT_BUILT      -4  std::runtime_error     (a call that needs a scene before build)
 * drape_cuda_last_error() returns the message of the last failing call on that handle (thread-local for NULL).
 *
 * Threading: one handle is driven by one host thread at a time (as the reference's sim thread drives its Solver,
 * sim_controller.cpp:57-98). Distinct handles are independent.
 */
#ifndef DRAPE_CUDA_H
#define DRAPE_CUDA_H

#include "drape_scene.h"

#ifdef __cplusplus
extern "C" {
#endif

enum {
  DRAPE_OK = 0,
  DRAPE_INVALID = -1,
  DRAPE_OUT_OF_RANGE = -2,
  DRAPE_DEVICE_ERROR = -3,
  DRAPE_NOT_BUILT = -4
};

typedef struct drape_solver drape_solver;

/* Library version (major * 10000 + minor * 100 + patch). */
int drape_cuda_version(void);

/* isAvailable(SolverBackend) (solver_factory.cpp:25-47): 1 when a CUDA device of compute capability 10.0 is present
   and this library's kernels load on it, else 0. */
int drape_cuda_is_available(void);

/* makeSolver (solver_factory.cpp:49-61): creates a solver on CUDA device `device`. Fails with DRAPE_DEVICE_ERROR
   ("cuda: ...") when the device is missing or is not sm_100. */
int drape_cuda_create(int device, drape_solver** out);
void drape_cuda_destroy(drape_solver* s);
const char* drape_cuda_last_error(const drape_solver* s);

/* Solver::build (solver.hpp:88): copies everything from the scene (the body field's samples too); a rebuild
   replaces all state. The block-CSR pattern, slot maps and term lists are built once here on the host in the
   reference's order (sim_model.cpp:41-175), then uploaded. */
int drape_cuda_build(drape_solver* s, const drape_scene_desc* scene);

/* Solver::updateFabric (solver.hpp:89): `count` must equal the garment's piece count. */
int drape_cuda_update_fabric(drape_solver* s, const char* garment, const drape_fabric* piece_fabric, uint32_t count);

/* Solver::setPhase (solver.hpp:90): DRAPE_PHASE_ASSEMBLING or DRAPE_PHASE_SETTLING. Entering Assembling resets the
   garment's assembly clock and re-measures its seams' start gaps (sim_model.cpp:295-305). */
int drape_cuda_set_phase(drape_solver* s, const char* garment, int phase);

/* Solver::step (solver.hpp:91; StepInput solver.hpp:57-61): max(1, substeps) implicit-Euler substeps of dt/substeps,
   each minimised by max(1, iterations) Newton iterations. Returns after the work has completed on the device. */
int drape_cuda_step(drape_solver* s, double dt, int substeps, int iterations);

/* Solver::readPositions (solver.hpp:92): 3 floats per particle; count must equal the particle count. */
int drape_cuda_read_positions(const drape_solver* s, float* out, size_t count);
/* Velocities, 3 floats per particle (part of Solver::snapshot). */
int drape_cuda_read_velocities(const drape_solver* s, float* out, size_t count);

/* Solver::stats (solver.hpp:93; SimModel::stats sim_model.cpp:222-241), reduced on the device in FP64. */
int drape_cuda_stats(drape_solver* s, drape_stats* out);

/* Solver::snapshot / restore (solver.hpp:94-95; Snapshot solver.hpp:76-83; sim_model.cpp:243-274).
   positions, velocities: 3 floats per particle; phases, assembly_time: per garment; seam_start_gap: per seam spring;
   contact_force: per particle. drape_cuda_snapshot_sizes gives the counts. restore throws invalid_argument when the
   particle or garment count does not match; a contact-force or seam array of another size is ignored (forces reset
   to zero, start gaps kept), as the reference does. */
int drape_cuda_snapshot_sizes(const drape_solver* s, uint32_t* particles, uint32_t* garments, uint32_t* seams);
int drape_cuda_snapshot(const drape_solver* s, float* positions, float* velocities, int32_t* phases,
                        double* assembly_time, float* seam_start_gap, double* contact_force);
int drape_cuda_restore(drape_solver* s, const float* positions, const float* velocities, uint32_t particles,
                       const int32_t* phases, const double* assembly_time, uint32_t garments,
                       const float* seam_start_gap, uint32_t seams, const double* contact_force,
                       uint32_t contact_count);

/* Solver::range / particleCount (solver.hpp:96-97). */
int drape_cuda_range(const drape_solver* s, const char* garment, uint32_t* offset, uint32_t* count);
int drape_cuda_particle_count(const drape_solver* s, size_t* out);

/* drapeToRest (libs/sim/include/drape/sim/drape_runner.hpp:40, libs/sim/src/drape_session.cpp:32-95): runs the
   Assembling -> Settling -> Settled frame loop with the stability guard, snapshots (kept on the device) and retries,
   for the listed garments. options may be NULL for the defaults of DrapeOptions. */
int drape_cuda_drape_to_rest(drape_solver* s, const char* const* garments, uint32_t garment_count,
                             const drape_drape_options* options, drape_drape_result* out);

/* Work counters (Newton, PCG, line-search halvings) since the last reset. */
int drape_cuda_counters(const drape_solver* s, drape_counters* out);
int drape_cuda_reset_counters(drape_solver* s);

/* PCG iterations of each Newton iteration since the last reset, oldest first (at most `capacity`; *count gets the
   number written). */
int drape_cuda_cg_history(const drape_solver* s, int32_t* out, size_t capacity, size_t* count);

/* The CUDA stream (a cudaStream_t) all of this solver's work runs on, for callers that time it with events. */
int drape_cuda_stream(const drape_solver* s, void** stream);

/* Kernel timing: with profiling on, every launch is bracketed by CUDA events on the solver's stream and its device
   time accumulated per kernel: [0] begin (predict + contact setup), [1] activate, [2] assemble, [3] solve
   (persistent PCG + line search), [4] finish, [5] stats. */
enum { DRAPE_KERNEL_COUNT = 7 };
typedef struct drape_profile {
  int64_t launches[DRAPE_KERNEL_COUNT];
  double milliseconds[DRAPE_KERNEL_COUNT];
  int64_t cg_iterations;        /* PCG iterations inside the profiled solve launches */
  int64_t energy_evaluations;   /* FP64 energy passes (E(0) and every line-search trial) */
} drape_profile;
/* enable: 0 off, 1 every kernel, 2 k_solve only (two events a launch, for timing a drape with little overhead);
   enabling also clears the accumulated figures. */
int drape_cuda_profile(drape_solver* s, int enable);
int drape_cuda_profile_read(const drape_solver* s, drape_profile* out);

/* Bytes copied host -> device and device -> host by this solver since creation. */
int drape_cuda_transfer_bytes(const drape_solver* s, uint64_t* h2d, uint64_t* d2h);

/* Block-CSR structure and term lists as built (the bit-exact artefacts of sim_model.cpp:41-175). sizes: [0] particles,
   [1] block slots, [2] stretch terms, [3] hinges, [4] seam springs. Pointers may be NULL. */
int drape_cuda_structure_sizes(const drape_solver* s, uint32_t sizes[5]);
int drape_cuda_structure(const drape_solver* s, uint32_t* row_start, uint32_t* col_index, uint32_t* diag_slot,
                         uint32_t* stretch_slots, uint32_t* hinge_slots, uint32_t* seam_slots, uint32_t* stretch_v,
                         uint32_t* hinge_v, uint32_t* seam_ab);

/* The same structure built on the host alone, without a device (for callers and tests that check the integer
   artefacts on machines without a GPU). */
typedef struct drape_model drape_model;
int drape_model_build(const drape_scene_desc* scene, drape_model** out);
void drape_model_destroy(drape_model* m);
const char* drape_model_last_error(void);
int drape_model_structure_sizes(const drape_model* m, uint32_t sizes[5]);
int drape_model_structure(const drape_model* m, uint32_t* row_start, uint32_t* col_index, uint32_t* diag_slot,
                          uint32_t* stretch_slots, uint32_t* hinge_slots, uint32_t* seam_slots, uint32_t* stretch_v,
                          uint32_t* hinge_v, uint32_t* seam_ab);
/* The assembly's gather lists, in place of the reference's per-particle and per-slot gather lists
   (gpu_solver_core.cpp:184-224): per particle its incidence entries (term kind << 30 | term << 2 | vertex a) in
   gather order; per off-diagonal block slot, in slot order, the slot (row << 6 | row-local position) and its
   contributions (incidence entry << 2 | block b of the entry's term) in gather order. sizes: particles, incidence
   entries, off-diagonal slots, contributions. Any output pointer may be null. */
int drape_model_gather_sizes(const drape_model* m, uint32_t sizes[4]);
int drape_model_gather_lists(const drape_model* m, uint32_t* inc_start, uint32_t* inc_entry, uint32_t* off_slot,
                             uint32_t* off_start, uint32_t* off_contrib);

/* Contact candidates (kernels.h:55-82 / cpu_solver.cpp:247-263) for given substep-start positions (3 floats per
   particle), computed by the device's contact-setup code path: near flag, normal (3 floats), plane offset. The solver
   state is not changed. */
int drape_cuda_contact_candidates(drape_solver* s, const float* x_start, uint8_t* near_flag, float* normal,
                                  float* offset);

/* The first Newton system of the next substep of length h (predict, contact setup and activation, term evaluation
   and assembly: cpu_solver.cpp:230-265 / gpu_solver_core.cpp:333-343), computed on the device without changing the
   solver state: blocks (9 floats per slot, row-major), gradient (3 floats per particle), contact-active flags. */
int drape_cuda_capture_system(drape_solver* s, double h, float* blocks, float* grad, uint8_t* active);

/* Contact-filtered block-Jacobi PCG (cpu_solver.cpp:169-213, kernels.h:237-347) on a system given in host memory,
   solved by the device's persistent PCG kernel: blocks 9 floats per slot (row-major), grad and normals 3 floats per
   particle. Returns the step, the unfiltered residual and the iteration count. */
int drape_cuda_pcg(uint32_t n, const uint32_t* row_start, const uint32_t* col_index, const float* blocks,
                   const uint8_t* pinned, const uint8_t* active, const float* normals, const float* grad,
                   int max_iterations, double tolerance, float* step, float* resid, int* iterations);

/* Block-CSR SpMV on device buffers (the PCG's inner product, kernels.h:272-289 without the contact filter):
   y = A x over rows and columns whose pinned flag is 0. Blocks are 9 planes of `slots_padded` floats (plane k holds
   component k = 3 * row + col of every slot); x and y are float4 per particle. Runs on `stream` (a cudaStream_t, or
   NULL for the legacy default stream) and does not synchronise. Used to measure the SpMV on its own. */
int drape_cuda_spmv_device(uint32_t n, const uint32_t* d_row_start, const uint32_t* d_col_index,
                           const float* d_blocks, uint32_t slots_padded, const uint8_t* d_pinned, const void* d_x,
                           void* d_y, void* stream);

/* The PCG of drape_cuda_pcg on a system that is already in device memory, allocating nothing. It is for callers that
   cannot allocate device memory: a host whose device memory is budgeted by another framework's pool allocator (an
   allocation outside the pool breaks its accounting), and frame-paced simulation loops that may not call
   cudaMalloc/cudaFree (cudaFree synchronises the whole device and either call can take unbounded time). This entry
   point has no counterpart in the reference.
   All of the solver's scratch (work vectors, preconditioner, converted flags, reduction partials, barrier state)
   lives in one file-scope device array of DRAPE_PCG_NOALLOC_SCRATCH_BYTES, which every GPU that loads the library
   holds until the process exits. Systems are limited to n <= DRAPE_PCG_NOALLOC_MAX_PARTICLES particles and
   slots <= DRAPE_PCG_NOALLOC_MAX_SLOTS block slots; larger ones are rejected with DRAPE_INVALID.
   Inputs and outputs are the caller's device buffers: row_start (n + 1) and col_index (slots = row_start[n], passed
   by value as `slots`) as u32; blocks as 9 planes of slots_padded floats (component 3 * row + col); pinned and
   active as one u8 per particle (active may be NULL); normals, grad, step and resid as float4 per particle (normals
   may be NULL). The iteration count is written to *d_iterations in device memory: -1 if the bounded grid barrier
   gave up, -2 if the device-side structure check refused the system (row_start not non-decreasing from 0 to
   `slots`, a column index >= n, or a row without its diagonal block; the allocating entry point throws for the
   same cases). Nothing is solved then and step/resid are left as they were. The work is queued on `stream` (a
   cudaStream_t, NULL for the legacy default stream) without synchronising; the return value reports argument and
   launch errors (slots < n is refused on the host).
   The first call on a device does a one-time set-up for that device (it looks up the array's device address with
   the device current); make that first call before any stream capture. Later calls made outside a capture look the
   address up again, so a re-created context is picked up. Every call shares the one array, which keeps
   the last call's contents; each call clears what must start at zero. Calls whose work overlaps on the GPU (other
   streams, other host threads, other devices' calls on the same device) race on the array: serialise them. */
#define DRAPE_PCG_NOALLOC_MAX_PARTICLES 8192u
#define DRAPE_PCG_NOALLOC_MAX_SLOTS 131072u
#define DRAPE_PCG_NOALLOC_SCRATCH_BYTES 2146560u
int drape_cuda_pcg_noalloc(uint32_t n, uint32_t slots, const uint32_t* d_row_start, const uint32_t* d_col_index,
                           const float* d_blocks, uint32_t slots_padded, const uint8_t* d_pinned,
                           const uint8_t* d_active, const void* d_normals, const void* d_grad, int max_iterations,
                           double tolerance, void* d_step, void* d_resid, int32_t* d_iterations, void* stream);

/* Measurement hook (no reference counterpart): device timestamps (%globaltimer, ns) of the frames run in batches
   (drape_cuda_drape_to_rest) since the last call: begin = the frame's first kernel, end = the end of its statistics
   kernel. end - begin is the frame's device-side duration; the next frame's begin minus this end is the device's idle
   time between them. Writes min(capacity, recorded) pairs, sets *count, and clears the record. */
int drape_cuda_frame_times(drape_solver* s, uint64_t* begin_ns, uint64_t* end_ns, size_t capacity, size_t* count);

/* Measurement hook (no reference counterpart): host seconds of the last drape_cuda_drape_to_rest, out[0] its set-up
   (the phase change and the first snapshot), out[1] its frame loop, out[2] the rest of the call. */
int drape_cuda_runner_host_seconds(const drape_solver* s, double* out);

/* How the host waits for the solver's stream (no reference counterpart): it polls for up to `spin_microseconds`, then
   sleeps 20 us between polls (default 200; UINT32_MAX polls without sleeping). Results do not depend on it. */
int drape_cuda_set_host_wait(drape_solver* s, uint32_t spin_microseconds);

/* The block-Jacobi PCG's form (no reference counterpart; each solves the reference's contact-filtered system with its
   stopping tests, cpu_solver.cpp:169-213): 0 (the default) the reference's order, two grid-wide reductions per
   iteration, run over resident rows (one 512-thread block per SM, each row's PCG state in its thread's registers, the
   block's matrix in a sliced layout in shared memory) where every block has at most 512 rows and its sliced matrix fits
   in shared memory, else on one 1024-thread block per SM: the two kernels give bit-identical results; 1 pipelined
   (Ghysels and Vanroose 2014), one reduction per iteration and three more work vectors, its FP32 recurrences drifting
   further from the products they stand for; 2 Chronopoulos-Gear, one reduction and one plain barrier per iteration
   with the reference order's recurrences; 3 the reference's order on the 1024-thread kernel whatever the scene (for
   comparison). Forms 0-2 give the same iterates in exact arithmetic and round differently. The learned preconditioner
   always runs its own PCG. */
int drape_cuda_set_pcg_variant(drape_solver* s, int variant);
/* Threads per block of the built scene's solve kernel under the current settings: 512 when the reference-order PCG runs
   over resident rows, else 1024 (the grid has one block per SM either way). */
int drape_cuda_solve_threads(const drape_solver* s, int* threads);

/* The bounded wait of the device grid barrier, in nanoseconds (0 restores the default of 2 s). A kernel whose barrier
   waits longer sets the handle's error status and returns instead of hanging; the step then fails with
   DRAPE_DEVICE_ERROR and the solver stays usable. */
int drape_cuda_set_barrier_limit(drape_solver* s, uint64_t nanoseconds);
/* Measurement hook (no reference counterpart): the synchronisation floor of the persistent solve on `device`: the
   solve's grid (one 1024-thread block per SM, cooperative) runs `iterations` rounds of grid-wide exchanges with no
   other work and *ns_per_iteration gets the device time per round (%globaltimer, block 0). mode 0: the two FP64 grid
   reductions of a reference-order PCG iteration; 1: one three-value reduction plus a plain barrier; 2: one three-value
   reduction; 3: two plain barriers; 4-7: modes 0-3 on one 512-thread block per SM (the resident-row form's grid). */
int drape_cuda_reduction_floor(int device, int mode, int iterations, double* ns_per_iteration);
/* Test hook: runs a grid barrier that can only end by its time limit (it waits for one more block than it has) on
   `blocks` blocks with the given limit, and returns the status the blocks read back in *status (0: released, which
   cannot happen; 1: timed out). Exercises the bounded wait without a device fault. */
int drape_cuda_test_barrier_timeout(int device, int blocks, uint64_t nanoseconds, int* status);
/* Test hook: make the next step fail with DRAPE_DEVICE_ERROR after `steps` more successful steps (-1: never), to
   exercise the caller's GPU -> CPU fallback (sim_controller.cpp:155-176) without a device fault. */
int drape_cuda_inject_failure(drape_solver* s, int steps);

#ifdef __cplusplus
}
#endif

#endif /* DRAPE_CUDA_H */
