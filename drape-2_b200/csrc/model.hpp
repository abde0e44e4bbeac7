// Host-side scene model of the CUDA solver: particles, energy terms, the block-CSR Hessian pattern with each term's
// slot map, the per-particle incidence lists and the per-slot contribution lists the assembly kernel walks.
//
// Restates drape::sim::SimModel (libs/sim/src/sim_model.hpp:20-83, sim_model.cpp:12-274) without Eigen. The integer
// artefacts (hinge order, rowStart / colIndex / diagSlot, stretchSlots / hingeSlots / seamSlots) are built with sorts
// instead of the reference's std::map and per-row vectors, and must equal the reference's bit for bit:
//   - hinges in lexicographic (min, max) edge order, each edge's triangles in insertion order (= std::map iteration,
//     sim_model.cpp:124-146), then per garment the seam springs interleaved with their seam hinges
//     (sim_model.cpp:147-175);
//   - rows = sorted unique coupled columns (self + every term's vertex set), each term's slots = the positions of its
//     vertices' columns in their rows (sim_model.cpp:35-74).
#pragma once

#include <array>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/drape_scene.h"

namespace drape_b200 {

inline constexpr double kContactReach = 0.01;   // sim_model.hpp:14
inline constexpr double kContactSnap = 0.0005;  // sim_model.hpp:15
inline constexpr uint32_t kMaxRowSlots = 64;    // the assembly kernel's per-row slot capacity

struct Vec3d {
  double x = 0, y = 0, z = 0;
};
struct Vec3f {
  float x = 0, y = 0, z = 0;
};

struct Model {
  struct Garment {
    std::string id;
    uint32_t offset = 0, count = 0;
    int phase = DRAPE_PHASE_SETTLING;
    double assemblyTime = 0;
    uint32_t fabricOffset = 0, pieceCount = 0;
  };
  struct HingeSide {
    uint32_t fabric = 0;
    double edgeDir[2] = {1, 0}, grain[2] = {0, 1};
  };
  struct Stretch {
    std::array<uint32_t, 3> v{};
    double dmInv[2][2] = {{1, 0}, {0, 1}};
    double area = 0;
    uint32_t fabric = 0;
  };
  struct Hinge {
    std::array<uint32_t, 4> v{};
    double K = 0, restAngle = 0;
  };
  struct Seam {
    uint32_t a = 0, b = 0, garment = 0;
    float startGap = 0;
  };

  drape_settings settings{};
  bool hasBody = false;
  drape_field_desc field{};      // values = nullptr; the samples are fieldData()[0, fieldCount)
  std::vector<float> fieldValues;  // the model's own copy of the samples (build with copyField), else empty
  const float* fieldSource = nullptr;  // without a copy: the caller's samples, valid while the build call runs
  std::size_t fieldCount = 0;          // samples in the field (0: no body)
  const float* fieldData() const { return fieldValues.empty() ? fieldSource : fieldValues.data(); }
  std::vector<Garment> garments;
  std::vector<drape_fabric> fabrics;
  std::vector<Vec3f> x, v;
  std::vector<double> mass, vertexArea;
  std::vector<Vec3d> fExt;
  std::vector<uint32_t> pFabric, pGarment;
  std::vector<uint8_t> pinned;
  std::vector<std::pair<uint32_t, Vec3f>> pins;
  std::vector<Stretch> stretch;
  std::vector<Hinge> hinges;
  std::vector<std::array<HingeSide, 2>> hingeSides;
  std::vector<double> hingeGeom;
  std::vector<Seam> seams;
  std::vector<uint32_t> rowStart, colIndex, diagSlot;
  // The off-diagonal slots in slot order (row << 6 | row-local position) and, per such slot k, the contributions
  // [offStart[k], offStart[k + 1]) of offContrib in gather order: incidence entry e << 2 | block b of its term.
  std::vector<uint32_t> offSlot, offStart, offContrib;
  // offContrib resolved for the device: per contribution, kind << 30 | term << 4 | vertex a << 2 | block b (the term's
  // entry and the block it adds), so the assembly reads the term's record without the incidence-entry indirection.
  std::vector<uint32_t> offCode;
  std::vector<std::array<uint32_t, 9>> stretchSlots;
  std::vector<std::array<uint32_t, 16>> hingeSlots;
  std::vector<std::array<uint32_t, 4>> seamSlots;
  std::vector<double> contactForce;

  // Incidence lists: for particle i, entries [incStart[i], incStart[i+1]) in the reference's gather order (stretch
  // (t, a) in term order, then hinges, then seams; gpu_solver_core.cpp:184-224). Entry code: kind << 30 | term << 2 | a
  // (kind 0 stretch, 1 hinge, 2 seam); incLocal packs the N row-local slot positions slots[a*N + b] - rowStart[i],
  // 8 bits each.
  std::vector<uint32_t> incStart, incEntry, incLocal;
  uint32_t maxRowSlots = 0, maxRowEntries = 0;

  // Throws invalid_argument / out_of_range like sim_model.cpp. Without copyField the model keeps no copy of the
  // collision field: fieldSource points at the scene's samples, which the caller uploads before the scene goes away.
  static Model build(const drape_scene_desc& scene, bool copyField = true);
  void updateFabric(const std::string& id, const drape_fabric* pieceFabric, uint32_t count);
  void setPhase(const std::string& id, int phase);
  std::size_t garmentIndex(const std::string& id) const;  // throws std::out_of_range for unknown ids
  double hingeStiffness(std::size_t hgi) const;
  void updateMass(uint32_t i);
  uint32_t slot(uint32_t row, uint32_t col) const;

 private:
  template <class F>
  void forEachTerm(F&& f) const;
  int termVertices(uint32_t code, uint32_t ab[4]) const;
  static int entryArity(uint32_t code);
  void buildIncidence();  // entry codes; then buildStructure: rows, slot maps, row-local slot positions
  void buildStructure();
};

}  // namespace drape_b200
