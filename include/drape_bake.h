/*
 * Collision-field bake on the GPU (libdrape_cuda.so): the signed distance field of the union of closed triangle
 * meshes, sampled on a regular grid, as drape::avatar::bakeCollisionField (libs/avatar/src/collision_bake.cpp:98-208,
 * libs/avatar/include/drape/avatar/collision_bake.hpp:10-20) makes it for the solver's body (SimScene::body).
 *
 * Per component: every triangle visits the samples of its bounding box grown by the band, keeping per sample the
 * nearest triangle (squared distance in FP64; ties go to the lower triangle index, as the reference's serial loop
 * keeps the first) and the sign from the angle-weighted pseudonormal of the nearest feature; samples farther than
 * the band are outside when connected to the grid boundary through other such samples (a flood fill), inside
 * otherwise; values are clamped to [-band, band]; components combine by minimum.
 *
 * Return codes follow include/drape_cuda.h; drape_bake_last_error() gives the message of this thread's last failing
 * call.
 */
#ifndef DRAPE_BAKE_H
#define DRAPE_BAKE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* drape::TriangleMesh (libs/core/include/drape/core/triangle_mesh.hpp): a closed manifold, triangles
   counter-clockwise seen from outside. */
typedef struct drape_mesh_desc {
  uint32_t vertex_count;
  const double* vertices;     /* 3 per vertex, metres */
  uint32_t triangle_count;
  const uint32_t* triangles;  /* 3 vertex indices per triangle */
} drape_mesh_desc;

/* drape::avatar::BakeOptions (collision_bake.hpp:10-14); defaults 0.004, 0.05, 0.02. */
typedef struct drape_bake_options {
  double cell_size;
  double padding;
  double band;
} drape_bake_options;

/* The grid the bake produces for these components (host only): origin = min corner of all vertices - padding,
   dims[a] = ceil((extent[a] + 2 padding) / cell_size) + 1 (collision_bake.cpp:99-117). Fails with DRAPE_INVALID
   when a component is not a closed manifold (isClosedManifold, libs/core/src/triangle_mesh.cpp:16-28). */
int drape_bake_grid(const drape_mesh_desc* components, uint32_t count, const drape_bake_options* options,
                    double origin[3], int32_t dims[3]);

/* bakeCollisionField on CUDA device `device`: writes value_count = dims[0] * dims[1] * dims[2] floats, x fastest
   (the CollisionField sample order, libs/core/include/drape/core/collision_field.hpp:16). The result equals the
   reference algorithm's in FP64 arithmetic rounded to float. */
int drape_bake_field(int device, const drape_mesh_desc* components, uint32_t count, const drape_bake_options* options,
                     float* values, size_t value_count);

/* Device time of the last drape_bake_field call on this thread, in milliseconds (its kernels, from the first to the
   last; the host's pseudonormal set-up and the final copy to `values` are outside it). */
double drape_bake_last_ms(void);
const char* drape_bake_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* DRAPE_BAKE_H */
