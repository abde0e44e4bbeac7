/*
 * ORACLE — test infrastructure only.
 *
 * C entry points of the CPU restatement of the reference cloth solver (cache25/drape-2, libs/sim). Only the tests,
 * the smoke check and the CPU-baseline leg of the benchmark load this library, and only as the checker: the product
 * path (libdrape_cuda) never links, loads or calls it.
 *
 * Two modes:
 *   faithful (full_fp64 = 0): particle positions and velocities stored as float, solve in double, exactly as
 *     drape::sim::CpuSolver (libs/sim/include/drape/sim/cpu_solver.hpp:11-13, libs/sim/src/cpu_solver.cpp:34-338);
 *   full FP64 (full_fp64 = 1): the same algorithm with double particle state and double push-out, the FP64 oracle
 *     the mixed-precision GPU path is measured against.
 *
 * Pinning: the term math, field sampling, push-out and block-Jacobi PCG are checked against the reference's own FP32
 * kernel bodies (libs/sim/kernels/kernels.h, term_math.h) compiled from the reference sources into oracle/_ref, and
 * the whole solver against the reference's analytic known-answer tests (libs/sim/tests/test_cpu_solver.cpp,
 * test_body_collision.cpp, test_seams.cpp, test_bending.cpp, test_friction.cpp, test_stretch.cpp). FP64 bit-level
 * parity with the Eigen build of the reference is unpinned: Eigen 3.4 is not available here.
 */
#ifndef DRAPE_ORACLE_API_H
#define DRAPE_ORACLE_API_H

#include "../include/drape_bake.h"
#include "../include/drape_scene.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_solver oracle_solver;

/* Return codes: 0 ok, -1 std::invalid_argument, -2 std::out_of_range, -3 other error. */
oracle_solver* oracle_create(int full_fp64);
void oracle_destroy(oracle_solver* s);
/* Host threads of the oracle's parallel loops (<= 0: all processors). Every count gives bit-identical results: each
   per-slot and per-particle sum keeps the serial scatter's order and every energy and dot-product sum is serial. */
void oracle_set_threads(int threads);
int oracle_threads(void);
const char* oracle_last_error(const oracle_solver* s);

int oracle_build(oracle_solver* s, const drape_scene_desc* scene);
int oracle_step(oracle_solver* s, double dt, int substeps, int iterations);
int oracle_set_phase(oracle_solver* s, const char* garment, int phase);
int oracle_update_fabric(oracle_solver* s, const char* garment, const drape_fabric* fabrics, uint32_t count);
int oracle_range(const oracle_solver* s, const char* garment, uint32_t* offset, uint32_t* count);
size_t oracle_particle_count(const oracle_solver* s);
int oracle_read_positions(const oracle_solver* s, double* out, size_t count);  /* 3 doubles per particle */
int oracle_read_velocities(const oracle_solver* s, double* out, size_t count); /* 3 doubles per particle */
int oracle_stats(const oracle_solver* s, drape_stats* out);
int oracle_counters(const oracle_solver* s, drape_counters* out);
void oracle_reset_counters(oracle_solver* s);

/* Snapshot (solver.hpp:76-83): positions/velocities 3 floats per particle; phases and assembly time per garment;
   seam start gaps per seam spring; contact force per particle. */
int oracle_snapshot_sizes(const oracle_solver* s, uint32_t* particles, uint32_t* garments, uint32_t* seams);
int oracle_snapshot(const oracle_solver* s, float* positions, float* velocities, int32_t* phases,
                    double* assembly_time, float* seam_start_gap, double* contact_force);
int oracle_restore(oracle_solver* s, const float* positions, const float* velocities, uint32_t particles,
                   const int32_t* phases, const double* assembly_time, uint32_t garments, const float* seam_start_gap,
                   uint32_t seams, const double* contact_force, uint32_t contact_count);

/* Sizes: [0] particles, [1] block slots, [2] stretch terms, [3] hinges, [4] seam springs, [5] gradient
   contributions, [6] block contributions. */
int oracle_structure_sizes(const oracle_solver* s, uint32_t sizes[7]);
/* Block-CSR pattern and the per-term slot maps (sim_model.cpp:41-74), the term vertex lists in build order
   (sim_model.cpp:107-175), and the fixed-order gather lists of the GPU solver (gpu_solver_core.cpp:184-224). Any
   pointer may be NULL. */
int oracle_structure(const oracle_solver* s, uint32_t* row_start, uint32_t* col_index, uint32_t* diag_slot,
                     uint32_t* stretch_slots, uint32_t* hinge_slots, uint32_t* seam_slots, uint32_t* stretch_v,
                     uint32_t* hinge_v, uint32_t* seam_ab, uint32_t* grad_start, uint32_t* grad_idx,
                     uint32_t* block_start, uint32_t* block_idx);
/* Per-term constants: stretch dmInv (4 per term: (0,0),(1,0),(0,1),(1,1)) and area; hinge K; particle mass. */
int oracle_term_constants(const oracle_solver* s, double* stretch_dm_inv, double* stretch_area, double* hinge_k,
                          double* mass);

/* The contact candidates of the next substep's setup (cpu_solver.cpp:247-263) for positions x (3 per particle):
   near flag, normal (3) and plane offset per particle. */
int oracle_contact_candidates(const oracle_solver* s, const double* x, uint8_t* near_flag, double* normal,
                              double* offset);

/* Runs the setup of a substep of length h and the first Newton evaluation (cpu_solver.cpp:230-265) on a copy of the
   state and returns the linear system the first solveLinear sees: blocks (9 doubles, row-major, per slot), grad
   (3 per particle), contact-active flags and normals. The solver state is not changed. */
int oracle_capture_system(const oracle_solver* s, double h, double* blocks, double* grad, uint8_t* active,
                          double* normals, double* energy);

/* Term math (energies.cpp, stretch.hpp, bending.hpp). Hessians are N*N blocks of 9 doubles, row-major. */
void oracle_eval_stretch(const double x[9], const double dm_inv[4], double area, const drape_fabric* f,
                         double limit_scale, double* energy, double grad[9], double hess[81]);
void oracle_eval_hinge(const double x[12], double k, double rest_angle, double* energy, double grad[12],
                       double hess[144]);
void oracle_eval_seam(const double x[6], double target, double k, double* energy, double grad[6], double hess[36]);
void oracle_eval_friction(const double x[3], const double x0[3], const double n[3], double mu_lambda, double eps,
                          double* energy, double grad[3], double hess[9]);
double oracle_dihedral(const double x[12], double grad[12]);
void oracle_bending_coefficients(double bend_warp, double bend_weft, double* p, double* q);
double oracle_edge_bend_stiffness(double p, double q, const double edge_dir[2], const double grain[2]);

/* CollisionField (collision_field.cpp:8-41) and the push-out helpers (collision.cpp:5-34). */
double oracle_field_sample(const drape_field_desc* f, const double p[3]);
void oracle_field_gradient(const drape_field_desc* f, const double p[3], double g[3]);
void oracle_collide_body(const drape_field_desc* f, float radius, float friction, const float x_prev[3], float x[3]);
void oracle_land_on_body(const drape_field_desc* f, float radius, const float from[3], const float to[3],
                         float out[3]);

/* Contact-filtered block-Jacobi PCG of CpuSolver::solveLinear (cpu_solver.cpp:169-213) on a given system. blocks:
   9 doubles per slot (row-major). Returns the step, the unfiltered residual and the iteration count. */
int oracle_pcg(uint32_t n, const uint32_t* row_start, const uint32_t* col_index, const double* blocks,
               const uint8_t* pinned, const uint8_t* active, const double* normals, const double* grad,
               int max_iterations, double tolerance, double* step, double* resid, int* iterations);

/* bakeCollisionField restated serially (bake_impl.hpp): bakes, keeps the field for oracle_bake_values, returns the
   grid. -1 (invalid_argument) for an open component. */
int oracle_bake(const drape_mesh_desc* components, uint32_t count, const drape_bake_options* options, double origin[3],
                int32_t dims[3]);
int oracle_bake_values(float* values, size_t count);
const char* oracle_bake_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* DRAPE_ORACLE_API_H */
