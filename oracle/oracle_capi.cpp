// ORACLE — test infrastructure only (see oracle_api.h). C entry points over oracle_impl.hpp.
#include "oracle_impl.hpp"
#include "bake_impl.hpp"

#include <omp.h>

// ---------------------------------------------------------------------------------------------------------------
// C API.

struct oracle_solver {
  oracle::Solver solver;
  bool fp64 = false;
  std::string error;
};

namespace {

template <class F>
int guarded(oracle_solver* s, F&& f) {
  try {
    f();
    if (s) s->error.clear();
    return 0;
  } catch (const std::invalid_argument& e) {
    if (s) s->error = e.what();
    return -1;
  } catch (const std::out_of_range& e) {
    if (s) s->error = e.what();
    return -2;
  } catch (const std::exception& e) {
    if (s) s->error = e.what();
    return -3;
  }
}

void requireBuilt(const oracle_solver* s) {
  if (!s) throw std::invalid_argument("null solver");
  if (!s->solver.built) throw std::runtime_error("solver not built");
}

void copyM3(const oracle::M3& a, double* out) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) out[3 * i + j] = a.m[i][j];
}

oracle::V3d load3(const double* p) { return {p[0], p[1], p[2]}; }
void store3(oracle::V3d v, double* p) {
  p[0] = v.x;
  p[1] = v.y;
  p[2] = v.z;
}

}  // namespace

extern "C" {

oracle_solver* oracle_create(int full_fp64) {
  auto* s = new oracle_solver;
  s->fp64 = full_fp64 != 0;
  return s;
}

void oracle_destroy(oracle_solver* s) { delete s; }

// Host threads of the oracle's parallel loops (results are identical for every count).
void oracle_set_threads(int threads) { omp_set_num_threads(threads > 0 ? threads : omp_get_num_procs()); }
int oracle_threads(void) { return omp_get_max_threads(); }

const char* oracle_last_error(const oracle_solver* s) { return s ? s->error.c_str() : "null solver"; }

int oracle_build(oracle_solver* s, const drape_scene_desc* scene) {
  return guarded(s, [&] {
    if (!s || !scene) throw std::invalid_argument("null argument");
    oracle::Solver next;
    next.m = oracle::Model::build(*scene, s->fp64);
    next.allocate();
    next.built = true;
    s->solver = std::move(next);
  });
}

int oracle_step(oracle_solver* s, double dt, int substeps, int iterations) {
  return guarded(s, [&] {
    requireBuilt(s);
    s->solver.advance(dt, substeps, iterations);
  });
}

int oracle_set_phase(oracle_solver* s, const char* garment, int phase) {
  return guarded(s, [&] {
    requireBuilt(s);
    s->solver.m.setPhase(garment ? garment : "", phase == 0 ? oracle::Assembling : oracle::Settling);
  });
}

int oracle_update_fabric(oracle_solver* s, const char* garment, const drape_fabric* fabrics, uint32_t count) {
  return guarded(s, [&] {
    requireBuilt(s);
    s->solver.m.updateFabric(garment ? garment : "", fabrics, count);
  });
}

int oracle_range(const oracle_solver* s, const char* garment, uint32_t* offset, uint32_t* count) {
  return guarded(const_cast<oracle_solver*>(s), [&] {
    requireBuilt(s);
    const auto& g = s->solver.m.garments[s->solver.m.garmentIndex(garment ? garment : "")];
    *offset = g.offset;
    *count = g.count;
  });
}

size_t oracle_particle_count(const oracle_solver* s) { return s && s->solver.built ? s->solver.m.x.size() : 0; }

int oracle_read_positions(const oracle_solver* s, double* out, size_t count) {
  return guarded(const_cast<oracle_solver*>(s), [&] {
    requireBuilt(s);
    if (count != s->solver.m.x.size()) throw std::invalid_argument("readPositions: span size must equal particleCount()");
    for (size_t i = 0; i < count; ++i) store3(s->solver.m.x[i], out + 3 * i);
  });
}

int oracle_read_velocities(const oracle_solver* s, double* out, size_t count) {
  return guarded(const_cast<oracle_solver*>(s), [&] {
    requireBuilt(s);
    if (count != s->solver.m.v.size()) throw std::invalid_argument("span size must equal particleCount()");
    for (size_t i = 0; i < count; ++i) store3(s->solver.m.v[i], out + 3 * i);
  });
}

int oracle_stats(const oracle_solver* s, drape_stats* out) {
  return guarded(const_cast<oracle_solver*>(s), [&] {
    requireBuilt(s);
    *out = s->solver.m.stats();
  });
}

int oracle_counters(const oracle_solver* s, drape_counters* out) {
  if (!s || !out) return -1;
  *out = s->solver.counters;
  return 0;
}

void oracle_reset_counters(oracle_solver* s) {
  if (s) s->solver.counters = drape_counters{};
}

int oracle_snapshot_sizes(const oracle_solver* s, uint32_t* particles, uint32_t* garments, uint32_t* seams) {
  return guarded(const_cast<oracle_solver*>(s), [&] {
    requireBuilt(s);
    *particles = static_cast<uint32_t>(s->solver.m.x.size());
    *garments = static_cast<uint32_t>(s->solver.m.garments.size());
    *seams = static_cast<uint32_t>(s->solver.m.seams.size());
  });
}

int oracle_snapshot(const oracle_solver* s, float* positions, float* velocities, int32_t* phases,
                    double* assembly_time, float* seam_start_gap, double* contact_force) {
  return guarded(const_cast<oracle_solver*>(s), [&] {
    requireBuilt(s);
    const auto& m = s->solver.m;
    for (size_t i = 0; i < m.x.size(); ++i) {
      const auto xf = oracle::tof(m.x[i]);
      const auto vf = oracle::tof(m.v[i]);
      positions[3 * i] = xf.x;
      positions[3 * i + 1] = xf.y;
      positions[3 * i + 2] = xf.z;
      velocities[3 * i] = vf.x;
      velocities[3 * i + 1] = vf.y;
      velocities[3 * i + 2] = vf.z;
      contact_force[i] = m.contactForce[i];
    }
    for (size_t g = 0; g < m.garments.size(); ++g) {
      phases[g] = m.garments[g].phase;
      assembly_time[g] = m.garments[g].assemblyTime;
    }
    for (size_t k = 0; k < m.seams.size(); ++k) seam_start_gap[k] = m.seams[k].startGap;
  });
}

int oracle_restore(oracle_solver* s, const float* positions, const float* velocities, uint32_t particles,
                   const int32_t* phases, const double* assembly_time, uint32_t garments, const float* seam_start_gap,
                   uint32_t seams, const double* contact_force, uint32_t contact_count) {
  return guarded(s, [&] {
    requireBuilt(s);
    auto& m = s->solver.m;
    if (particles != m.x.size() || garments != m.garments.size())
      throw std::invalid_argument("snapshot does not match this scene");
    for (size_t i = 0; i < particles; ++i) {
      m.x[i] = {positions[3 * i], positions[3 * i + 1], positions[3 * i + 2]};
      m.v[i] = {velocities[3 * i], velocities[3 * i + 1], velocities[3 * i + 2]};
    }
    if (contact_count == m.contactForce.size()) {
      for (size_t i = 0; i < contact_count; ++i) m.contactForce[i] = contact_force[i];
    } else {
      std::fill(m.contactForce.begin(), m.contactForce.end(), 0.0);
    }
    for (size_t g = 0; g < garments; ++g) {
      m.garments[g].phase = phases[g] == 0 ? oracle::Assembling : oracle::Settling;
      m.garments[g].assemblyTime = assembly_time[g];
    }
    if (seams == m.seams.size())
      for (size_t k = 0; k < seams; ++k) m.seams[k].startGap = seam_start_gap[k];
  });
}

int oracle_structure_sizes(const oracle_solver* s, uint32_t sizes[7]) {
  return guarded(const_cast<oracle_solver*>(s), [&] {
    requireBuilt(s);
    const auto& m = s->solver.m;
    const auto n = static_cast<uint32_t>(m.x.size());
    const auto S = static_cast<uint32_t>(m.stretch.size()), H = static_cast<uint32_t>(m.hinges.size()),
               K = static_cast<uint32_t>(m.seams.size());
    sizes[0] = n;
    sizes[1] = static_cast<uint32_t>(m.colIndex.size());
    sizes[2] = S;
    sizes[3] = H;
    sizes[4] = K;
    sizes[5] = n + 3 * S + 4 * H + 2 * K;
    sizes[6] = n + 9 * S + 16 * H + 4 * K;
  });
}

int oracle_structure(const oracle_solver* s, uint32_t* row_start, uint32_t* col_index, uint32_t* diag_slot,
                     uint32_t* stretch_slots, uint32_t* hinge_slots, uint32_t* seam_slots, uint32_t* stretch_v,
                     uint32_t* hinge_v, uint32_t* seam_ab, uint32_t* grad_start, uint32_t* grad_idx,
                     uint32_t* block_start, uint32_t* block_idx) {
  return guarded(const_cast<oracle_solver*>(s), [&] {
    requireBuilt(s);
    const auto& m = s->solver.m;
    const auto n = static_cast<uint32_t>(m.x.size());
    const auto S = static_cast<uint32_t>(m.stretch.size()), H = static_cast<uint32_t>(m.hinges.size()),
               K = static_cast<uint32_t>(m.seams.size());
    const auto B = static_cast<uint32_t>(m.colIndex.size());
    if (row_start) std::copy(m.rowStart.begin(), m.rowStart.end(), row_start);
    if (col_index) std::copy(m.colIndex.begin(), m.colIndex.end(), col_index);
    if (diag_slot) std::copy(m.diagSlot.begin(), m.diagSlot.end(), diag_slot);
    for (uint32_t t = 0; t < S; ++t) {
      if (stretch_slots) std::copy(m.stretchSlots[t].begin(), m.stretchSlots[t].end(), stretch_slots + 9 * t);
      if (stretch_v) std::copy(m.stretch[t].v.begin(), m.stretch[t].v.end(), stretch_v + 3 * t);
    }
    for (uint32_t h = 0; h < H; ++h) {
      if (hinge_slots) std::copy(m.hingeSlots[h].begin(), m.hingeSlots[h].end(), hinge_slots + 16 * h);
      if (hinge_v) std::copy(m.hinges[h].v.begin(), m.hinges[h].v.end(), hinge_v + 4 * h);
    }
    for (uint32_t k = 0; k < K; ++k) {
      if (seam_slots) std::copy(m.seamSlots[k].begin(), m.seamSlots[k].end(), seam_slots + 4 * k);
      if (seam_ab) {
        seam_ab[2 * k] = m.seams[k].a;
        seam_ab[2 * k + 1] = m.seams[k].b;
      }
    }
    // Gather lists in the GPU solver's fixed order: the particle's own term, then stretch, hinge and seam terms in
    // term order (gpu_solver_core.cpp:184-224).
    if (grad_start || grad_idx || block_start || block_idx) {
      std::vector<std::vector<uint32_t>> g(n), b(B);
      for (uint32_t i = 0; i < n; ++i) {
        g[i].push_back(i);
        b[m.diagSlot[i]].push_back(i);
      }
      for (uint32_t t = 0; t < S; ++t)
        for (uint32_t a = 0; a < 3; ++a) {
          g[m.stretch[t].v[a]].push_back(n + 3 * t + a);
          for (uint32_t c = 0; c < 3; ++c) b[m.stretchSlots[t][3 * a + c]].push_back(n + 9 * t + 3 * a + c);
        }
      for (uint32_t h = 0; h < H; ++h)
        for (uint32_t a = 0; a < 4; ++a) {
          g[m.hinges[h].v[a]].push_back(n + 3 * S + 4 * h + a);
          for (uint32_t c = 0; c < 4; ++c) b[m.hingeSlots[h][4 * a + c]].push_back(n + 9 * S + 16 * h + 4 * a + c);
        }
      for (uint32_t k = 0; k < K; ++k) {
        const uint32_t vs[2] = {m.seams[k].a, m.seams[k].b};
        for (uint32_t a = 0; a < 2; ++a) {
          g[vs[a]].push_back(n + 3 * S + 4 * H + 2 * k + a);
          for (uint32_t c = 0; c < 2; ++c) b[m.seamSlots[k][2 * a + c]].push_back(n + 9 * S + 16 * H + 4 * k + 2 * a + c);
        }
      }
      auto flatten = [](const std::vector<std::vector<uint32_t>>& lists, uint32_t* start, uint32_t* idx) {
        uint32_t pos = 0;
        if (start) start[0] = 0;
        for (std::size_t l = 0; l < lists.size(); ++l) {
          for (auto v : lists[l]) {
            if (idx) idx[pos] = v;
            ++pos;
          }
          if (start) start[l + 1] = pos;
        }
      };
      flatten(g, grad_start, grad_idx);
      flatten(b, block_start, block_idx);
    }
  });
}

int oracle_term_constants(const oracle_solver* s, double* stretch_dm_inv, double* stretch_area, double* hinge_k,
                          double* mass) {
  return guarded(const_cast<oracle_solver*>(s), [&] {
    requireBuilt(s);
    const auto& m = s->solver.m;
    for (size_t t = 0; t < m.stretch.size(); ++t) {
      const auto& d = m.stretch[t].dmInv.d;
      if (stretch_dm_inv) {
        stretch_dm_inv[4 * t] = d[0][0];
        stretch_dm_inv[4 * t + 1] = d[1][0];
        stretch_dm_inv[4 * t + 2] = d[0][1];
        stretch_dm_inv[4 * t + 3] = d[1][1];
      }
      if (stretch_area) stretch_area[t] = m.stretch[t].area;
    }
    if (hinge_k)
      for (size_t h = 0; h < m.hinges.size(); ++h) hinge_k[h] = m.hinges[h].K;
    if (mass)
      for (size_t i = 0; i < m.mass.size(); ++i) mass[i] = m.mass[i];
  });
}

int oracle_contact_candidates(const oracle_solver* s, const double* x, uint8_t* near_flag, double* normal,
                              double* offset) {
  return guarded(const_cast<oracle_solver*>(s), [&] {
    requireBuilt(s);
    const auto& m = s->solver.m;
    for (size_t i = 0; i < m.x.size(); ++i) {
      near_flag[i] = 0;
      store3(oracle::V3d{}, normal + 3 * i);
      offset[i] = 0;
      if (!m.hasBody || m.pinned[i]) continue;
      const oracle::V3d xs = load3(x + 3 * i);
      const double radius = m.contactRadius(i);
      const double phi = m.body.sample(xs);
      if (phi >= radius + oracle::kContactReach) continue;
      const oracle::V3d nrm = m.body.gradient(xs);
      if (oracle::isZero(nrm)) continue;
      near_flag[i] = 1;
      store3(nrm, normal + 3 * i);
      offset[i] = radius - phi;
    }
  });
}

int oracle_capture_system(const oracle_solver* s, double h, double* blocks, double* grad, uint8_t* active,
                          double* normals, double* energy) {
  return guarded(const_cast<oracle_solver*>(s), [&] {
    requireBuilt(s);
    oracle::Solver copy = s->solver;
    copy.beginSubstep(h);
    const double e = copy.evaluateWithContact(1.0 / (h * h));
    if (energy) *energy = e;
    for (size_t k = 0; k < copy.blocks.size(); ++k)
      if (blocks) copyM3(copy.blocks[k], blocks + 9 * k);
    for (size_t i = 0; i < copy.grad.size(); ++i) {
      if (grad) store3(copy.grad[i], grad + 3 * i);
      if (active) active[i] = copy.contactActive[i];
      if (normals) store3(copy.contactNormal[i], normals + 3 * i);
    }
  });
}

void oracle_eval_stretch(const double x[9], const double dm_inv[4], double area, const drape_fabric* f,
                         double limit_scale, double* energy, double grad[9], double hess[81]) {
  oracle::Dm dm;
  dm.d[0][0] = dm_inv[0];
  dm.d[1][0] = dm_inv[1];
  dm.d[0][1] = dm_inv[2];
  dm.d[1][1] = dm_inv[3];
  oracle::V3d xs[3] = {load3(x), load3(x + 3), load3(x + 6)};
  oracle::TermEval<3> te;
  oracle::evalStretchTerm(dm, area, xs, oracle::fabricFrom(*f), limit_scale, te);
  *energy = te.energy;
  for (int a = 0; a < 3; ++a) {
    store3(te.grad[a], grad + 3 * a);
    for (int b = 0; b < 3; ++b) copyM3(te.hess[a][b], hess + 9 * (3 * a + b));
  }
}

void oracle_eval_hinge(const double x[12], double k, double rest_angle, double* energy, double grad[12],
                       double hess[144]) {
  oracle::V3d xs[4] = {load3(x), load3(x + 3), load3(x + 6), load3(x + 9)};
  oracle::TermEval<4> te;
  oracle::evalHingeTerm(k, rest_angle, xs, te);
  *energy = te.energy;
  for (int a = 0; a < 4; ++a) {
    store3(te.grad[a], grad + 3 * a);
    for (int b = 0; b < 4; ++b) copyM3(te.hess[a][b], hess + 9 * (4 * a + b));
  }
}

void oracle_eval_seam(const double x[6], double target, double k, double* energy, double grad[6], double hess[36]) {
  oracle::V3d xs[2] = {load3(x), load3(x + 3)};
  oracle::TermEval<2> te;
  oracle::evalSeamTerm(xs, target, k, te);
  *energy = te.energy;
  for (int a = 0; a < 2; ++a) {
    store3(te.grad[a], grad + 3 * a);
    for (int b = 0; b < 2; ++b) copyM3(te.hess[a][b], hess + 9 * (2 * a + b));
  }
}

void oracle_eval_friction(const double x[3], const double x0[3], const double n[3], double mu_lambda, double eps,
                          double* energy, double grad[3], double hess[9]) {
  oracle::TermEval<1> te;
  oracle::evalFrictionTerm(load3(x), load3(x0), load3(n), mu_lambda, eps, te);
  *energy = te.energy;
  store3(te.grad[0], grad);
  copyM3(te.hess[0][0], hess);
}

double oracle_dihedral(const double x[12], double grad[12]) {
  oracle::V3d xs[4] = {load3(x), load3(x + 3), load3(x + 6), load3(x + 9)};
  oracle::V3d g[4];
  double theta = 0;
  oracle::evalDihedral(xs, theta, g);
  for (int a = 0; a < 4; ++a) store3(g[a], grad + 3 * a);
  return theta;
}

void oracle_bending_coefficients(double bend_warp, double bend_weft, double* p, double* q) {
  const auto c = oracle::bendingCoefficients(bend_warp, bend_weft);
  *p = c.p;
  *q = c.q;
}

double oracle_edge_bend_stiffness(double p, double q, const double edge_dir[2], const double grain[2]) {
  return oracle::edgeBendStiffness({p, q}, edge_dir, grain);
}

double oracle_field_sample(const drape_field_desc* f, const double p[3]) {
  return oracle::fieldFrom(f).sample(load3(p));
}

void oracle_field_gradient(const drape_field_desc* f, const double p[3], double g[3]) {
  store3(oracle::fieldFrom(f).gradient(load3(p)), g);
}

void oracle_collide_body(const drape_field_desc* f, float radius, float friction, const float x_prev[3], float x[3]) {
  const auto field = oracle::fieldFrom(f);
  oracle::V3f xf{x[0], x[1], x[2]};
  oracle::collideBodyF(field, radius, friction, {x_prev[0], x_prev[1], x_prev[2]}, xf);
  x[0] = xf.x;
  x[1] = xf.y;
  x[2] = xf.z;
}

void oracle_land_on_body(const drape_field_desc* f, float radius, const float from[3], const float to[3],
                         float out[3]) {
  const auto field = oracle::fieldFrom(f);
  const auto r = oracle::landOnBodyF(field, radius, {from[0], from[1], from[2]}, {to[0], to[1], to[2]});
  out[0] = r.x;
  out[1] = r.y;
  out[2] = r.z;
}

int oracle_pcg(uint32_t n, const uint32_t* row_start, const uint32_t* col_index, const double* blocks,
               const uint8_t* pinned, const uint8_t* active, const double* normals, const double* grad,
               int max_iterations, double tolerance, double* step, double* resid, int* iterations) {
  oracle_solver tmp;
  return guarded(&tmp, [&] {
    oracle::Solver s;
    s.m.pinned.assign(pinned, pinned + n);
    s.m.rowStart.assign(row_start, row_start + n + 1);
    const uint32_t B = row_start[n];
    s.m.colIndex.assign(col_index, col_index + B);
    s.m.diagSlot.resize(n);
    for (uint32_t i = 0; i < n; ++i) s.m.diagSlot[i] = s.m.slot(i, i);
    s.m.settings.maxCgIterations = max_iterations;
    s.m.settings.cgTolerance = tolerance;
    s.m.contactForce.assign(n, 0.0);
    s.m.x.assign(n, oracle::V3d{});
    s.allocate();
    for (uint32_t k = 0; k < B; ++k)
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) s.blocks[k].m[i][j] = blocks[9 * k + 3 * i + j];
    for (uint32_t i = 0; i < n; ++i) {
      s.grad[i] = load3(grad + 3 * i);
      s.contactActive[i] = active ? active[i] : 0;
      if (normals) s.contactNormal[i] = load3(normals + 3 * i);
    }
    s.solveLinear();
    for (uint32_t i = 0; i < n; ++i) {
      store3(s.step[i], step + 3 * i);
      store3(s.resid[i], resid + 3 * i);
    }
    *iterations = static_cast<int>(s.counters.cg_iterations);
  });
}

namespace {
thread_local obake::Field g_bake;
thread_local std::string g_bakeError;
}  // namespace

int oracle_bake(const drape_mesh_desc* components, uint32_t count, const drape_bake_options* options, double origin[3],
                int32_t dims[3]) {
  try {
    if (!components || !options || !origin || !dims) throw std::invalid_argument("null argument");
    std::vector<obake::Mesh> meshes(count);
    for (uint32_t c = 0; c < count; ++c) {
      const drape_mesh_desc& d = components[c];
      for (uint32_t i = 0; i < d.vertex_count; ++i)
        meshes[c].v.push_back({d.vertices[3 * i], d.vertices[3 * i + 1], d.vertices[3 * i + 2]});
      for (uint32_t t = 0; t < d.triangle_count; ++t) {
        const uint32_t* tr = d.triangles + 3ull * t;
        if (tr[0] >= d.vertex_count || tr[1] >= d.vertex_count || tr[2] >= d.vertex_count)
          throw std::invalid_argument("triangle vertex index out of range");
        meshes[c].t.push_back({tr[0], tr[1], tr[2]});
      }
    }
    g_bake = obake::bake(meshes, options->cell_size, options->padding, options->band);
    for (int a = 0; a < 3; ++a) {
      origin[a] = g_bake.origin[a];
      dims[a] = g_bake.dims[a];
    }
    return 0;
  } catch (const std::invalid_argument& e) {
    g_bakeError = e.what();
    return -1;
  } catch (const std::exception& e) {
    g_bakeError = e.what();
    return -3;
  }
}

int oracle_bake_values(float* values, size_t count) {
  if (!values || count != g_bake.values.size()) return -1;
  std::copy(g_bake.values.begin(), g_bake.values.end(), values);
  return 0;
}

const char* oracle_bake_last_error(void) { return g_bakeError.c_str(); }

}  // extern "C"
