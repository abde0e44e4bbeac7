// Conversion of a host Model (model.hpp) into the device records and launch parameters of kernels.cuh. Shared by the
// single solver (solver.cu) and the batch (batch.cu), so a garment's device data is the same in both.
#pragma once

#include <vector>

#include "kernels.cuh"
#include "model.hpp"

namespace dmodel {

using drape_b200::Model;

inline float4 f4(drape_b200::Vec3f v) { return make_float4(v.x, v.y, v.z, 0.0f); }

inline std::vector<dcu::Particle> particles(const Model& m) {
  std::vector<dcu::Particle> out(m.x.size());
  for (size_t i = 0; i < out.size(); ++i)
    out[i] = {static_cast<float>(m.mass[i]), m.pFabric[i], m.pGarment[i], m.pinned[i] ? 1u : 0u};
  return out;
}

inline std::vector<dcu::Fabric> fabrics(const Model& m) {
  std::vector<dcu::Fabric> out;
  for (const auto& f : m.fabrics) {
    dcu::Fabric d{};
    d.k[0] = static_cast<float>(f.stretch_warp);
    d.k[1] = static_cast<float>(f.stretch_weft);
    d.k[2] = static_cast<float>(f.stretch_bias);
    d.limit[0] = static_cast<float>(f.strain_limit_warp);
    d.limit[1] = static_cast<float>(f.strain_limit_weft);
    d.thickness = static_cast<float>(f.thickness);
    d.friction = static_cast<float>(f.friction);
    d.damping = static_cast<float>(f.damping);
    out.push_back(d);
  }
  if (out.empty()) out.push_back(dcu::Fabric{});
  return out;
}

inline std::vector<dcu::Garment> garments(const Model& m) {
  std::vector<dcu::Garment> out;
  for (const auto& g : m.garments) out.push_back({g.phase, 0, g.assemblyTime});
  if (out.empty()) out.push_back(dcu::Garment{});
  return out;
}

inline std::vector<dcu::Stretch> stretches(const Model& m) {
  std::vector<dcu::Stretch> out;
  for (const auto& t : m.stretch) {
    dcu::Stretch d{};
    for (int k = 0; k < 3; ++k) d.v[k] = t.v[k];
    d.fabric = t.fabric;
    d.d = make_float4(static_cast<float>(t.dmInv[0][0]), static_cast<float>(t.dmInv[1][0]),
                      static_cast<float>(t.dmInv[0][1]), static_cast<float>(t.dmInv[1][1]));
    d.area = static_cast<float>(t.area);
    out.push_back(d);
  }
  return out;
}

inline std::vector<dcu::Hinge> hinges(const Model& m) {
  std::vector<dcu::Hinge> out;
  for (const auto& h : m.hinges)
    out.push_back({{h.v[0], h.v[1], h.v[2], h.v[3]}, static_cast<float>(h.K), static_cast<float>(h.restAngle), {0, 0}});
  return out;
}

inline std::vector<dcu::Seam> seams(const Model& m) {
  std::vector<dcu::Seam> out;
  for (const auto& s : m.seams) out.push_back({s.a, s.b, s.garment, s.startGap});
  return out;
}

// Column indices with bit 31 set where the column's particle is pinned.
inline std::vector<uint32_t> columns(const Model& m) {
  std::vector<uint32_t> cols(m.colIndex);
  for (auto& c : cols)
    if (m.pinned[c]) c |= dcu::kPinnedBit;
  return cols;
}

// Initial x, v, external force and pin target per particle (float4).
inline void state(const Model& m, std::vector<float4>& xs, std::vector<float4>& vs, std::vector<float4>& fe,
                  std::vector<float4>& pp) {
  const size_t n = m.x.size();
  xs.assign(n, float4{});
  vs.assign(n, float4{});
  fe.assign(n, float4{});
  pp.assign(n, float4{});
  for (size_t i = 0; i < n; ++i) {
    xs[i] = f4(m.x[i]);
    vs[i] = f4(m.v[i]);
    fe[i] = make_float4(static_cast<float>(m.fExt[i].x), static_cast<float>(m.fExt[i].y),
                        static_cast<float>(m.fExt[i].z), 0.0f);
  }
  for (const auto& [i, pos] : m.pins) pp[i] = f4(pos);
}

// Launch parameters and field view of a model: everything of Dev except the device pointers and the per-launch
// substep length and solve sizes.
inline void params(const Model& m, uint32_t slotsPadded, unsigned long long barrierLimitNs, dcu::Dev& d) {
  auto& P = d.P;
  P.gravity[0] = static_cast<float>(m.settings.gravity[0]);
  P.gravity[1] = static_cast<float>(m.settings.gravity[1]);
  P.gravity[2] = static_cast<float>(m.settings.gravity[2]);
  P.limitScale = static_cast<float>(m.settings.strain_limit_stiffness_scale);
  P.seamStiffness = static_cast<float>(m.settings.seam_stiffness);
  P.closingSpeed = static_cast<float>(m.settings.assembly_closing_speed);
  P.frictionSlip = static_cast<float>(m.settings.friction_slip_speed);
  P.collisionOffset = static_cast<float>(m.settings.collision_offset);
  P.dampingScale = static_cast<float>(m.settings.damping_scale);
  P.assemblyExtraDamping = static_cast<float>(m.settings.assembly_extra_damping);
  P.contactReach = static_cast<float>(drape_b200::kContactReach);
  P.contactSnap = static_cast<float>(drape_b200::kContactSnap);
  P.cgTolerance = m.settings.cg_tolerance;
  P.maxCg = m.settings.max_cg_iterations;
  P.n = static_cast<uint32_t>(m.x.size());
  P.nStretch = static_cast<uint32_t>(m.stretch.size());
  P.nHinge = static_cast<uint32_t>(m.hinges.size());
  P.nSeam = static_cast<uint32_t>(m.seams.size());
  P.nBlocks = static_cast<uint32_t>(m.colIndex.size());
  P.nGarments = static_cast<uint32_t>(m.garments.size());
  P.slotsPadded = slotsPadded;
  P.barrierLimitNs = barrierLimitNs;
  d.field.present = m.fieldCount > 0 ? 1 : 0;
  d.field.ox = static_cast<float>(m.field.origin[0]);
  d.field.oy = static_cast<float>(m.field.origin[1]);
  d.field.oz = static_cast<float>(m.field.origin[2]);
  d.field.cell = static_cast<float>(m.field.cell_size);
  d.field.band = static_cast<float>(m.hasBody ? m.field.band : 0.02);
  for (int a = 0; a < 3; ++a) d.field.dims[a] = m.field.dims[a];
  for (int a = 0; a < 3; ++a) d.fieldOrigin[a] = m.field.origin[a];
  d.fieldCell = m.field.cell_size;
}

}  // namespace dmodel
