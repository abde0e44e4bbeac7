/* Pattern -> simulation mesh: the drape::garment::buildSimMesh path (libs/garment/src/sim_mesh_builder.cpp:196-323,
   libs/garment/include/drape/garment/sim_mesh_builder.hpp:10-20) as a C ABI. Host code only (no device): a grain-
   aligned hexagonal lattice inside each pattern piece, the piece outline sampled at corners and seam ends, a
   constrained Delaunay triangulation of both with the outline as constraint, Laplacian smoothing of the interior, and
   seam vertex pairs 1:1. The output arrays are exactly the garment arrays of drape_scene_desc (rest, vertex_piece,
   vertex_area, triangles, triangle_piece, piece_grain, seam_pairs), so a mesh goes straight into a solver. */
#ifndef DRAPE_MESH_H
#define DRAPE_MESH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One cubic Bezier segment of a piece outline: p0, p1, p2, p3 as (x, y) pairs, metres
   (libs/core/include/drape/core/bezier.hpp). */
typedef struct drape_bezier {
  double p[8];
} drape_bezier;

/* A pattern piece (libs/core/include/drape/core/pattern.hpp:44-55): a closed counter-clockwise outline of cubic
   segments, its grainline and fabric slot. */
typedef struct drape_piece_desc {
  const char* id;
  const drape_bezier* segments;
  uint32_t segment_count;
  double grain[2];
  const char* fabric_slot;
} drape_piece_desc;

/* A seam (pattern.hpp:58-72): two arc-length ranges [start, end] on piece outlines, one traversed reversed. */
typedef struct drape_seam_desc {
  const char* id;
  const char* piece_a;
  double start_a, end_a;
  int32_t reversed_a;
  const char* piece_b;
  double start_b, end_b;
  int32_t reversed_b;
  double ease;
} drape_seam_desc;

typedef struct drape_pattern_desc {
  const drape_piece_desc* pieces;
  uint32_t piece_count;
  const drape_seam_desc* seams;
  uint32_t seam_count;
} drape_pattern_desc;

typedef struct drape_mesh drape_mesh;

/* particleDistance (sim_mesh_builder.cpp:14-21): quality 0 Draft 0.020 m, 1 Standard 0.010 m, 2 Fine 0.005 m. */
double drape_mesh_particle_distance(int quality);

/* buildSimMesh(pattern, h) (sim_mesh_builder.hpp:19): returns DRAPE_INVALID (-1) with a message listing the
   validation rule ids ("outline-closed", "seam-range", ...) for an invalid pattern, as the reference's MeshError. */
int drape_mesh_build(const drape_pattern_desc* pattern, double particle_distance, drape_mesh** out);
void drape_mesh_destroy(drape_mesh* m);
const char* drape_mesh_last_error(void);
/* sizes: vertices, triangles, pieces, seam pairs. */
int drape_mesh_sizes(const drape_mesh* m, uint32_t sizes[4]);
/* SimMesh (libs/core/include/drape/core/sim_mesh.hpp:18-27): rest (2 per vertex), vertex_piece, boundary,
   vertex_area, triangles (3 per triangle, counter-clockwise), triangle_piece, piece_grain (2 per piece), seam_pairs
   (a, b, seam, index per pair). Any output pointer may be null. */
int drape_mesh_read(const drape_mesh* m, double* rest, uint32_t* vertex_piece, uint8_t* boundary, double* vertex_area,
                    uint32_t* triangles, uint32_t* triangle_piece, double* piece_grain, uint32_t* seam_pairs);

#ifdef __cplusplus
}
#endif

#endif
