/*
 * Plain-data description of a cloth scene, as the solver boundary receives it.
 *
 * Each struct restates one reference type field for field, with Eigen vectors flattened to double arrays and
 * std::vector members passed as pointer + count:
 *   drape_fabric          <- drape::FabricPhysical        (libs/core/include/drape/core/fabric.hpp:10-18)
 *   drape_garment_desc    <- drape::sim::SimGarment + SimMesh
 *                            (libs/sim/include/drape/sim/solver.hpp:32-37, libs/core/include/drape/core/sim_mesh.hpp:14-30)
 *   drape_field_desc      <- drape::CollisionField        (libs/core/include/drape/core/collision_field.hpp:11-20)
 *   drape_settings        <- drape::sim::SimSettings      (libs/sim/include/drape/sim/solver.hpp:19-30)
 *   drape_scene_desc      <- drape::sim::SimScene         (libs/sim/include/drape/sim/solver.hpp:49-55)
 *   drape_stats           <- drape::sim::SimStats         (libs/sim/include/drape/sim/solver.hpp:63-69)
 *   drape_drape_options   <- drape::sim::DrapeOptions     (libs/sim/include/drape/sim/drape_runner.hpp:14-26)
 *   drape_drape_result    <- drape::sim::DrapeResult      (libs/sim/include/drape/sim/drape_runner.hpp:28-37)
 *
 * No C++ types cross this header: it is valid C99 and C++.
 */
#ifndef DRAPE_SCENE_H
#define DRAPE_SCENE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct drape_fabric {
  double stretch_warp, stretch_weft, stretch_bias; /* N/m */
  double strain_limit_warp, strain_limit_weft;     /* fraction (0.05 = 5%) */
  double bend_warp, bend_weft;                     /* N m */
  double weight;                                   /* kg/m^2 */
  double thickness;                                /* m */
  double friction, damping;                        /* 0..1 */
} drape_fabric;

typedef struct drape_garment_desc {
  const char* id;                    /* garment id (NUL-terminated) */
  uint32_t vertex_count;             /* V */
  const double* rest;                /* 2V: pattern-space position (m) */
  const uint32_t* vertex_piece;      /* V: pattern piece index */
  const double* vertex_area;         /* V: 1/3 of incident triangle rest areas (m^2) */
  uint32_t triangle_count;           /* T */
  const uint32_t* triangles;         /* 3T: CCW in pattern space, garment-local vertex indices */
  const uint32_t* triangle_piece;    /* T */
  uint32_t piece_count;              /* P */
  const double* piece_grain;         /* 2P: unit grainline per piece */
  const drape_fabric* piece_fabric;  /* P */
  uint32_t seam_pair_count;          /* Q */
  const uint32_t* seam_pairs;        /* 4Q: a, b (garment-local vertices), seam, index; grouped by seam */
  const double* initial_positions;   /* 3V: world position (m) */
} drape_garment_desc;

typedef struct drape_field_desc {
  double origin[3];
  double cell_size;
  int32_t dims[3];
  double band;
  const float* values; /* dims[0]*dims[1]*dims[2] samples, x fastest; NULL with dims 0 = no samples */
} drape_field_desc;

typedef struct drape_settings {
  double gravity[3];                  /* default (0, -9.81, 0) */
  double collision_offset;            /* 0.003 m */
  double assembly_closing_speed;      /* 0.25 m/s */
  double assembly_extra_damping;      /* 10 1/s */
  double damping_scale;               /* 5 1/s */
  double strain_limit_stiffness_scale;/* 100 */
  double seam_stiffness;              /* 1e4 N/m */
  double friction_slip_speed;         /* 3e-4 m/s */
  int32_t max_cg_iterations;          /* 50 */
  double cg_tolerance;                /* 1e-2 relative residual */
} drape_settings;

typedef struct drape_scene_desc {
  uint32_t garment_count;
  const drape_garment_desc* garments;
  const drape_field_desc* body;       /* NULL: no body. The solver keeps its own copy of the samples. */
  uint32_t pin_count;
  const uint32_t* pin_particles;      /* global particle index */
  const double* pin_positions;        /* 3 per pin */
  uint32_t force_count;
  const uint32_t* force_particles;
  const double* forces;               /* 3 per force, newtons */
  drape_settings settings;
} drape_scene_desc;

typedef struct drape_stats {
  int32_t has_non_finite;
  double kinetic_energy;
  double rms_speed;
  double max_seam_gap;
  double max_body_penetration;
} drape_stats;

/* SimPhase order (solver.hpp:17). */
enum { DRAPE_PHASE_ASSEMBLING = 0, DRAPE_PHASE_SETTLING = 1 };

typedef struct drape_drape_options {
  int32_t substeps;            /* 1 */
  int32_t iterations;          /* 2 */
  double frame_dt;             /* 1/60 */
  double max_assembly_seconds; /* 3 */
  double seam_gap_done;        /* 0.001 */
  double settle_rms_speed;     /* 0.002 */
  int32_t settle_hold_frames;  /* 60 */
  double max_sim_seconds;      /* 20 */
  int32_t snapshot_every;      /* 30 */
  int32_t max_retries;         /* 3 */
  int32_t energy_rise_frames;  /* 60 */
  /* Frames the device runs per host wait (1 = the reference's one frame per wait; default 10). Not a reference option:
   * the runner replays a batch's discarded frames where a decision falls inside it, so every value gives the same
   * outcome, frame for frame. The learned preconditioner and the batch runner keep one wait per frame. */
  int32_t frames_per_wait;     /* 10 */
} drape_drape_options;

enum { DRAPE_STATE_ASSEMBLING = 0, DRAPE_STATE_SETTLING, DRAPE_STATE_SETTLED, DRAPE_STATE_FAILED, DRAPE_STATE_TIMED_OUT };

typedef struct drape_drape_result {
  int32_t settled;
  int32_t failed;
  double simulated_seconds;
  int32_t retries;
  int32_t frames_run;
  double assembly_end_seam_gap;
  double assembly_seconds;
} drape_drape_result;

/* Work counters of the Newton solver, summed over the calls since the last reset. */
typedef struct drape_counters {
  int64_t substeps;
  int64_t newton_iterations;
  int64_t cg_iterations;
  int64_t line_search_halvings;
  int64_t precond_fallbacks; /* learned preconditioner abandoned for block-Jacobi */
  int64_t learned_solves;    /* PCG solves that started with the learned preconditioner */
  int64_t pcg_nanoseconds;   /* device time inside the PCG solves (CG init to the last iteration; %globaltimer) */
} drape_counters;

#ifdef __cplusplus
}
#endif

#endif /* DRAPE_SCENE_H */
