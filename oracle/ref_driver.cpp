// ORACLE — test infrastructure only. Built by oracle/Makefile into oracle/_ref/libref_emulated.so together with the
// reference's own sources, compiled where they lie (never copied into this repository):
//   libs/sim/src/gpu/emulated_device.cpp, libs/sim/src/gpu/compute_device.cpp, and through them the FP32 kernel
//   bodies libs/sim/kernels/kernels.h, term_math.h, gpu_layout.h, gpu_compat.h.
// This file is a host driver over the reference's EmulatedDevice that issues the kernels in the order of the
// reference's GpuSolverCore (libs/sim/src/gpu/gpu_solver_core.cpp:142-407): the reference's 32-bit GPU algorithm run
// on the CPU, used as the known-answer oracle for the FP32 CUDA path (term math, contact candidates, PCG, and whole
// substeps on identical inputs). The model (particles, terms, slot maps) comes from the FP64 restatement in
// oracle_impl.hpp, since the reference's SimModel needs Eigen.
#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "gpu/emulated_device.hpp"
#include "gpu_layout.h"
#include "kernels.h"
#include "oracle_impl.hpp"

using drape::sim::BufferId;
using drape::sim::EmulatedDevice;
using drape::sim::Kernel;
using dgpu::uint;

namespace {

dgpu::float4 f4(oracle::V3d v) {
  return {static_cast<float>(v.x), static_cast<float>(v.y), static_cast<float>(v.z), 0.0f};
}

dgpu::GpuFabric gpuFabric(const oracle::Fabric& f) {
  dgpu::GpuFabric g{};
  g.stretchWarp = static_cast<float>(f.stretchWarp);
  g.stretchWeft = static_cast<float>(f.stretchWeft);
  g.stretchBias = static_cast<float>(f.stretchBias);
  g.strainLimitWarp = static_cast<float>(f.strainLimitWarp);
  g.strainLimitWeft = static_cast<float>(f.strainLimitWeft);
  g.weight = static_cast<float>(f.weight);
  g.thickness = static_cast<float>(f.thickness);
  g.friction = static_cast<float>(f.friction);
  g.damping = static_cast<float>(f.damping);
  return g;
}

dgpu::GpuFabric gpuFabric(const drape_fabric& f) { return gpuFabric(oracle::fabricFrom(f)); }

dgpu::FieldInfo fieldInfo(const drape_field_desc* f) {
  dgpu::FieldInfo info{};
  if (!f || !f->values) return info;
  info.origin = {static_cast<float>(f->origin[0]), static_cast<float>(f->origin[1]), static_cast<float>(f->origin[2]),
                 0.0f};
  for (int a = 0; a < 3; ++a) info.dims[a] = static_cast<uint>(f->dims[a]);
  info.cellSize = static_cast<float>(f->cell_size);
  info.band = static_cast<float>(f->band);
  return info;
}

struct Device {
  EmulatedDevice dev;
  template <class T>
  T* view(BufferId b) {
    return static_cast<T*>(dev.contents(b));
  }
  template <class T>
  BufferId upload(const std::vector<T>& data) {
    const BufferId b = dev.create(sizeof(T) * std::max<std::size_t>(data.size(), 1));
    if (!data.empty()) std::memcpy(dev.contents(b), data.data(), sizeof(T) * data.size());
    return b;
  }
  template <class T>
  void write(BufferId b, const std::vector<T>& data) {
    if (!data.empty()) std::memcpy(dev.contents(b), data.data(), sizeof(T) * data.size());
  }
  template <class T>
  BufferId array(std::size_t count) {
    return dev.create(sizeof(T) * std::max<std::size_t>(count, 1));
  }
  void dispatch(Kernel k, uint threads, std::initializer_list<BufferId> buffers) {
    dev.dispatch(k, threads, std::span<const BufferId>(buffers.begin(), buffers.size()));
  }
};

}  // namespace

struct ref_solver {
  Device d;
  oracle::Model m;
  bool built = false;
  std::string error;
  uint n = 0, nStretch = 0, nHinge = 0, nSeam = 0, nBlocks = 0, nEnergies = 0;
  BufferId particles, garments, fabrics, fExt, pinPos, stretch, hinges, seams, rowStart, colIndex, diagSlot;
  BufferId gradStart, gradIdx, blockStart, blockIdx, fieldValues, fieldInfoBuf;
  BufferId paramsDeriv, paramsEnergy, x, v, xStart, yRel, u, trialU, grad, step, r, z, p, ap, apFull, resid;
  BufferId precond, blocks, contact, energies, gradContrib, hessContrib, scalars, partials, prodA, prodB, moved;
  BufferId specRz, specR0, specPAp, specRr, specRzNew;
  drape_counters counters{};

  std::vector<dgpu::GpuParticle> particleData() const {
    std::vector<dgpu::GpuParticle> out(n);
    for (uint i = 0; i < n; ++i)
      out[i] = {static_cast<float>(m.mass[i]), m.pFabric[i], m.pGarment[i], m.pinned[i] ? 1u : 0u};
    return out;
  }
  std::vector<dgpu::GpuFabric> fabricData() const {
    std::vector<dgpu::GpuFabric> out;
    for (const auto& f : m.fabrics) out.push_back(gpuFabric(f));
    return out;
  }
  std::vector<dgpu::GpuGarment> garmentData() const {
    std::vector<dgpu::GpuGarment> out;
    for (const auto& g : m.garments)
      out.push_back({g.phase == oracle::Settling ? 1u : 0u, static_cast<float>(g.assemblyTime), {0, 0}});
    return out;
  }
  std::vector<dgpu::GpuHinge> hingeData() const {
    std::vector<dgpu::GpuHinge> out;
    for (const auto& h : m.hinges)
      out.push_back({{h.v[0], h.v[1], h.v[2], h.v[3]}, static_cast<float>(h.K), static_cast<float>(h.restAngle), {0, 0}});
    return out;
  }
  std::vector<dgpu::GpuSeam> seamData() const {
    std::vector<dgpu::GpuSeam> out;
    for (const auto& s : m.seams) out.push_back({s.a, s.b, s.garment, s.startGap});
    return out;
  }

  void syncToModel() {
    const auto* xs = d.view<dgpu::float4>(x);
    const auto* vs = d.view<dgpu::float4>(v);
    const auto* cs = d.view<dgpu::GpuContact>(contact);
    for (uint i = 0; i < n; ++i) {
      m.x[i] = {xs[i].x, xs[i].y, xs[i].z};
      m.v[i] = {vs[i].x, vs[i].y, vs[i].z};
      m.contactForce[i] = cs[i].force;
    }
  }
  void syncFromModel() {
    auto* xs = d.view<dgpu::float4>(x);
    auto* vs = d.view<dgpu::float4>(v);
    auto* cs = d.view<dgpu::GpuContact>(contact);
    for (uint i = 0; i < n; ++i) {
      xs[i] = f4(m.x[i]);
      vs[i] = f4(m.v[i]);
      cs[i].force = static_cast<float>(m.contactForce[i]);
    }
    d.write(particles, particleData());
    d.write(fabrics, fabricData());
    d.write(garments, garmentData());
    d.write(hinges, hingeData());
    d.write(seams, seamData());
  }

  void build(const drape_scene_desc& scene) {
    m = oracle::Model::build(scene, false);
    n = static_cast<uint>(m.x.size());
    nStretch = static_cast<uint>(m.stretch.size());
    nHinge = static_cast<uint>(m.hinges.size());
    nSeam = static_cast<uint>(m.seams.size());
    nBlocks = static_cast<uint>(m.colIndex.size());
    nEnergies = n + nStretch + nHinge + nSeam;
    const uint nGrad = n + 3 * nStretch + 4 * nHinge + 2 * nSeam;
    const uint nHess = n + 9 * nStretch + 16 * nHinge + 4 * nSeam;
    particles = d.upload(particleData());
    fabrics = d.upload(fabricData());
    garments = d.upload(garmentData());
    hinges = d.upload(hingeData());
    seams = d.upload(seamData());
    {
      std::vector<dgpu::float4> fe(n), pins(n);
      for (uint i = 0; i < n; ++i) fe[i] = f4(m.fExt[i]);
      for (const auto& [i, pos] : m.pins) pins[i] = f4(pos);
      fExt = d.upload(fe);
      pinPos = d.upload(pins);
    }
    {
      std::vector<dgpu::GpuStretch> st;
      for (const auto& t : m.stretch) {
        dgpu::GpuStretch g{};
        for (int k = 0; k < 3; ++k) g.v[k] = t.v[k];
        g.dmInv = {static_cast<float>(t.dmInv.d[0][0]), static_cast<float>(t.dmInv.d[1][0]),
                   static_cast<float>(t.dmInv.d[0][1]), static_cast<float>(t.dmInv.d[1][1])};
        g.area = static_cast<float>(t.area);
        g.fabric = t.fabric;
        st.push_back(g);
      }
      stretch = d.upload(st);
    }
    rowStart = d.upload(m.rowStart);
    colIndex = d.upload(m.colIndex);
    diagSlot = d.upload(m.diagSlot);
    {
      std::vector<std::vector<uint>> g(n), b(nBlocks);
      for (uint i = 0; i < n; ++i) {
        g[i].push_back(i);
        b[m.diagSlot[i]].push_back(i);
      }
      for (uint t = 0; t < nStretch; ++t)
        for (uint a = 0; a < 3; ++a) {
          g[m.stretch[t].v[a]].push_back(n + 3 * t + a);
          for (uint c = 0; c < 3; ++c) b[m.stretchSlots[t][3 * a + c]].push_back(n + 9 * t + 3 * a + c);
        }
      for (uint h = 0; h < nHinge; ++h)
        for (uint a = 0; a < 4; ++a) {
          g[m.hinges[h].v[a]].push_back(n + 3 * nStretch + 4 * h + a);
          for (uint c = 0; c < 4; ++c) b[m.hingeSlots[h][4 * a + c]].push_back(n + 9 * nStretch + 16 * h + 4 * a + c);
        }
      for (uint k = 0; k < nSeam; ++k) {
        const uint vs[2] = {m.seams[k].a, m.seams[k].b};
        for (uint a = 0; a < 2; ++a) {
          g[vs[a]].push_back(n + 3 * nStretch + 4 * nHinge + 2 * k + a);
          for (uint c = 0; c < 2; ++c)
            b[m.seamSlots[k][2 * a + c]].push_back(n + 9 * nStretch + 16 * nHinge + 4 * k + 2 * a + c);
        }
      }
      auto flatten = [](const std::vector<std::vector<uint>>& lists, std::vector<uint>& start, std::vector<uint>& idx) {
        start.assign(1, 0);
        for (const auto& l : lists) {
          idx.insert(idx.end(), l.begin(), l.end());
          start.push_back(static_cast<uint>(idx.size()));
        }
      };
      std::vector<uint> gs, gi, bs, bi;
      flatten(g, gs, gi);
      flatten(b, bs, bi);
      gradStart = d.upload(gs);
      gradIdx = d.upload(gi);
      blockStart = d.upload(bs);
      blockIdx = d.upload(bi);
    }
    {
      dgpu::FieldInfo info{};
      if (m.hasBody && !m.body.values.empty()) {
        info.origin = f4(m.body.origin);
        for (int a = 0; a < 3; ++a) info.dims[a] = static_cast<uint>(m.body.dims[a]);
        info.cellSize = static_cast<float>(m.body.cellSize);
        info.band = static_cast<float>(m.body.band);
        fieldValues = d.upload(m.body.values);
      } else {
        fieldValues = d.array<float>(1);
      }
      fieldInfoBuf = d.upload(std::vector<dgpu::FieldInfo>{info});
    }
    dgpu::StepParams sp{};
    sp.gravity = f4(m.settings.gravity);
    sp.limitScale = static_cast<float>(m.settings.strainLimitStiffnessScale);
    sp.seamStiffness = static_cast<float>(m.settings.seamStiffness);
    sp.closingSpeed = static_cast<float>(m.settings.assemblyClosingSpeed);
    sp.frictionSlip = static_cast<float>(m.settings.frictionSlipSpeed);
    sp.cgTolerance = static_cast<float>(m.settings.cgTolerance);
    sp.collisionOffset = static_cast<float>(m.settings.collisionOffset);
    sp.dampingScale = static_cast<float>(m.settings.dampingScale);
    sp.assemblyExtraDamping = static_cast<float>(m.settings.assemblyExtraDamping);
    sp.contactReach = static_cast<float>(oracle::kContactReach);
    sp.contactSnap = static_cast<float>(oracle::kContactSnap);
    sp.n = n;
    sp.nStretch = nStretch;
    sp.nHinge = nHinge;
    sp.nSeam = nSeam;
    sp.nBlocks = nBlocks;
    sp.maxCgIterations = static_cast<uint>(m.settings.maxCgIterations);
    sp.withDerivatives = 1;
    paramsDeriv = d.upload(std::vector<dgpu::StepParams>{sp});
    sp.withDerivatives = 0;
    paramsEnergy = d.upload(std::vector<dgpu::StepParams>{sp});
    x = d.array<dgpu::float4>(n);
    v = d.array<dgpu::float4>(n);
    for (BufferId* b : {&xStart, &yRel, &u, &trialU, &grad, &step, &r, &z, &p, &ap, &apFull, &resid})
      *b = d.array<dgpu::float4>(n);
    precond = d.array<dgpu::Block3>(n);
    blocks = d.array<dgpu::Block3>(nBlocks);
    contact = d.array<dgpu::GpuContact>(n);
    energies = d.array<float>(nEnergies);
    gradContrib = d.array<dgpu::float4>(nGrad);
    hessContrib = d.array<dgpu::Block3>(nHess);
    scalars = d.array<dgpu::CgScalars>(1);
    partials = d.array<float>(n / dgpu::kReduceBlock + 1);
    prodA = d.array<float>(n);
    prodB = d.array<float>(n);
    moved = d.array<float>(n);
    auto spec = [&](uint selector) { return d.upload(std::vector<dgpu::ReduceSpec>{{n, selector, {0, 0}}}); };
    specRz = spec(dgpu::kReduceRz);
    specR0 = spec(dgpu::kReduceR0);
    specPAp = spec(dgpu::kReducePAp);
    specRr = spec(dgpu::kReduceRr);
    specRzNew = spec(dgpu::kReduceRzNew);
    syncFromModel();
    built = true;
  }

  void reduce(BufferId spec, BufferId input) {
    d.dispatch(Kernel::ReducePartial, n / dgpu::kReduceBlock + 1, {spec, input, partials});
    d.dispatch(Kernel::ReduceFinal, 1, {spec, partials, scalars});
  }
  void evalTerms(BufferId params, BufferId positions) {
    d.dispatch(Kernel::InertiaFriction, n, {params, particles, fabrics, positions, yRel, contact, energies, gradContrib, hessContrib});
    d.dispatch(Kernel::StretchTerms, nStretch, {params, stretch, fabrics, xStart, positions, energies, gradContrib, hessContrib});
    d.dispatch(Kernel::HingeTerms, nHinge, {params, hinges, xStart, positions, energies, gradContrib, hessContrib});
    d.dispatch(Kernel::SeamTerms, nSeam, {params, seams, garments, xStart, positions, energies, gradContrib, hessContrib});
  }
  double energySum() {
    const float* e = d.view<float>(energies);
    double s = 0;
    for (uint k = 0; k < nEnergies; ++k) s += e[k];
    return s;
  }
  void cgIteration() {
    d.dispatch(Kernel::Spmv, n, {paramsDeriv, particles, rowStart, colIndex, blocks, contact, scalars, p, apFull, ap, prodA});
    reduce(specPAp, prodA);
    d.dispatch(Kernel::CgAlpha, 1, {scalars});
    d.dispatch(Kernel::CgUpdate, n, {paramsDeriv, scalars, p, ap, apFull, step, r, resid, prodB});
    reduce(specRr, prodB);
    d.dispatch(Kernel::CgCheck, 1, {paramsDeriv, scalars});
    d.dispatch(Kernel::CgPrecond, n, {paramsDeriv, contact, scalars, precond, r, z, prodA});
    reduce(specRzNew, prodA);
    d.dispatch(Kernel::CgBeta, 1, {scalars});
    d.dispatch(Kernel::CgDirection, n, {paramsDeriv, scalars, z, p});
  }

  void substep(double h, int iterations) {
    for (BufferId b : {paramsDeriv, paramsEnergy}) {
      auto* sp = d.view<dgpu::StepParams>(b);
      sp->h = static_cast<float>(h);
      sp->invH2 = static_cast<float>(1.0 / (h * h));
    }
    auto* lineParams = d.view<dgpu::StepParams>(paramsEnergy);
    ++counters.substeps;
    d.dev.begin();
    d.dispatch(Kernel::Predict, n, {paramsDeriv, particles, garments, x, v, fExt, xStart, yRel, u});
    d.dispatch(Kernel::ContactSetup, n, {paramsDeriv, particles, fabrics, xStart, fieldValues, fieldInfoBuf, contact});
    for (int it = 0; it < iterations; ++it) {
      if (it > 0) d.dev.begin();
      ++counters.newton_iterations;
      d.dispatch(Kernel::ContactActivate, n, {paramsDeriv, contact, u});
      evalTerms(paramsDeriv, u);
      d.dispatch(Kernel::GatherGrad, n, {paramsDeriv, particles, gradStart, gradIdx, gradContrib, grad});
      d.dispatch(Kernel::GatherBlocks, nBlocks, {paramsDeriv, blockStart, blockIdx, hessContrib, blocks});
      d.dispatch(Kernel::ContactRelease, n, {paramsDeriv, contact, grad});
      d.dev.submitAndWait();
      const double e0 = energySum();
      d.dev.begin();
      d.dispatch(Kernel::Precondition, n, {paramsDeriv, particles, diagSlot, blocks, precond});
      d.dispatch(Kernel::CgInit, n, {paramsDeriv, contact, precond, grad, step, resid, r, z, p, prodA, prodB});
      reduce(specRz, prodA);
      reduce(specR0, prodB);
      const int maxCg = m.settings.maxCgIterations;
      for (int c = 0; c < maxCg; ++c) cgIteration();
      d.dispatch(Kernel::ContactForce, n, {paramsDeriv, contact, resid});
      d.dev.submitAndWait();
      counters.cg_iterations += d.view<dgpu::CgScalars>(scalars)->iteration;
      double slope = 0;
      {
        const auto* g = d.view<dgpu::float4>(grad);
        const auto* s = d.view<dgpu::float4>(step);
        for (uint i = 0; i < n; ++i)
          slope += static_cast<double>(g[i].x) * s[i].x + static_cast<double>(g[i].y) * s[i].y +
                   static_cast<double>(g[i].z) * s[i].z;
      }
      if (!(slope < 0)) break;
      double alpha = 1.0;
      for (int ls = 0; ls < 20; ++ls) {
        lineParams->alpha = static_cast<float>(alpha);
        d.dev.begin();
        d.dispatch(Kernel::TrialPositions, n, {paramsEnergy, u, step, trialU});
        evalTerms(paramsEnergy, trialU);
        d.dev.submitAndWait();
        if (energySum() <= e0 + 1e-4 * alpha * slope) break;
        alpha *= 0.5;
        ++counters.line_search_halvings;
      }
      lineParams->alpha = static_cast<float>(alpha);
      d.dev.begin();
      d.dispatch(Kernel::ApplyStep, n, {paramsEnergy, contact, u, step, moved});
      d.dev.submitAndWait();
      const float* mv = d.view<float>(moved);
      double maxMove = 0;
      for (uint i = 0; i < n; ++i) maxMove = std::max(maxMove, static_cast<double>(mv[i]));
      if (maxMove < 1e-9) break;
    }
    d.dev.begin();
    d.dispatch(Kernel::FinishSubstep, n,
               {paramsDeriv, particles, fabrics, garments, xStart, u, pinPos, fieldValues, fieldInfoBuf, x, v});
    d.dev.submitAndWait();
    for (auto& g : m.garments)
      if (g.phase == oracle::Assembling) g.assemblyTime += h;
    d.write(garments, garmentData());
  }
};

namespace {

template <class F>
int guarded(ref_solver* s, F&& f) {
  try {
    f();
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

void need(const ref_solver* s) {
  if (!s || !s->built) throw std::runtime_error("not built");
}

dgpu::Block3 blockFromRowMajor(const float* b) {
  dgpu::Block3 out{};
  out.c0 = {b[0], b[3], b[6], 0.0f};
  out.c1 = {b[1], b[4], b[7], 0.0f};
  out.c2 = {b[2], b[5], b[8], 0.0f};
  return out;
}

void storeMat(const dgpu::Mat3& m, float* out) {  // row-major
  const dgpu::float3 c[3] = {m.c0, m.c1, m.c2};
  for (int col = 0; col < 3; ++col) {
    out[0 * 3 + col] = c[col].x;
    out[1 * 3 + col] = c[col].y;
    out[2 * 3 + col] = c[col].z;
  }
}

}  // namespace

extern "C" {

ref_solver* ref_create(void) { return new ref_solver; }
void ref_destroy(ref_solver* s) { delete s; }
const char* ref_last_error(const ref_solver* s) { return s ? s->error.c_str() : "null"; }

int ref_build(ref_solver* s, const drape_scene_desc* scene) {
  return guarded(s, [&] {
    if (!s || !scene) throw std::invalid_argument("null argument");
    s->d = Device{};
    s->built = false;
    s->counters = drape_counters{};
    s->build(*scene);
  });
}

int ref_step(ref_solver* s, double dt, int substeps, int iterations) {
  return guarded(s, [&] {
    need(s);
    if (s->n == 0) return;
    const int sub = std::max(1, substeps);
    const double h = dt / sub;
    const int its = std::max(1, iterations);
    for (int k = 0; k < sub; ++k) s->substep(h, its);
  });
}

int ref_set_phase(ref_solver* s, const char* garment, int phase) {
  return guarded(s, [&] {
    need(s);
    s->syncToModel();
    s->m.setPhase(garment ? garment : "", phase == 0 ? oracle::Assembling : oracle::Settling);
    s->syncFromModel();
  });
}

int ref_read_positions(ref_solver* s, double* out, size_t count) {
  return guarded(s, [&] {
    need(s);
    if (count != s->n) throw std::invalid_argument("size mismatch");
    const auto* xs = s->d.view<dgpu::float4>(s->x);
    for (uint i = 0; i < s->n; ++i) {
      out[3 * i] = xs[i].x;
      out[3 * i + 1] = xs[i].y;
      out[3 * i + 2] = xs[i].z;
    }
  });
}

int ref_stats(ref_solver* s, drape_stats* out) {
  return guarded(s, [&] {
    need(s);
    s->syncToModel();
    *out = s->m.stats();
  });
}

int ref_counters(const ref_solver* s, drape_counters* out) {
  if (!s || !out) return -1;
  *out = s->counters;
  return 0;
}

/* Runs the reference's k_contact_setup on given substep-start positions (3 floats per particle) and returns the near
   flags, normals (3 floats) and plane offsets. */
int ref_contact_setup(ref_solver* s, const float* x_start, uint8_t* near_flag, float* normal, float* offset) {
  return guarded(s, [&] {
    need(s);
    auto* xs = s->d.view<dgpu::float4>(s->xStart);
    for (uint i = 0; i < s->n; ++i) xs[i] = {x_start[3 * i], x_start[3 * i + 1], x_start[3 * i + 2], 0.0f};
    s->d.dev.begin();
    s->d.dispatch(Kernel::ContactSetup, s->n,
                  {s->paramsDeriv, s->particles, s->fabrics, s->xStart, s->fieldValues, s->fieldInfoBuf, s->contact});
    s->d.dev.submitAndWait();
    auto* cs = s->d.view<dgpu::GpuContact>(s->contact);
    for (uint i = 0; i < s->n; ++i) {
      near_flag[i] = cs[i].nearBody ? 1 : 0;
      normal[3 * i] = cs[i].normal.x;
      normal[3 * i + 1] = cs[i].normal.y;
      normal[3 * i + 2] = cs[i].normal.z;
      offset[i] = cs[i].normal.w;
      cs[i] = dgpu::GpuContact{};
    }
  });
}

void ref_eval_stretch(const float x[9], const float dm_inv[4], float area, const drape_fabric* f, float limit_scale,
                      float* energy, float grad[9], float hess[81]) {
  dgpu::GpuStretch t{};
  t.dmInv = {dm_inv[0], dm_inv[1], dm_inv[2], dm_inv[3]};
  t.area = area;
  dgpu::float3 xs[3] = {{x[0], x[1], x[2]}, {x[3], x[4], x[5]}, {x[6], x[7], x[8]}};
  dgpu::TermEvalF<3> te;
  dgpu::clearTerm(te);
  dgpu::evalStretchF(t, xs, gpuFabric(*f), limit_scale, te);
  *energy = te.energy;
  for (int a = 0; a < 3; ++a) {
    grad[3 * a] = te.grad[a].x;
    grad[3 * a + 1] = te.grad[a].y;
    grad[3 * a + 2] = te.grad[a].z;
    for (int b = 0; b < 3; ++b) storeMat(te.hess[a][b], hess + 9 * (3 * a + b));
  }
}

void ref_eval_hinge(const float x[12], float k, float rest_angle, float* energy, float grad[12], float hess[144]) {
  dgpu::GpuHinge t{};
  t.K = k;
  t.restAngle = rest_angle;
  dgpu::float3 xs[4] = {{x[0], x[1], x[2]}, {x[3], x[4], x[5]}, {x[6], x[7], x[8]}, {x[9], x[10], x[11]}};
  dgpu::TermEvalF<4> te;
  dgpu::clearTerm(te);
  dgpu::evalHingeF(t, xs, te);
  *energy = te.energy;
  for (int a = 0; a < 4; ++a) {
    grad[3 * a] = te.grad[a].x;
    grad[3 * a + 1] = te.grad[a].y;
    grad[3 * a + 2] = te.grad[a].z;
    for (int b = 0; b < 4; ++b) storeMat(te.hess[a][b], hess + 9 * (4 * a + b));
  }
}

void ref_eval_seam(const float x[6], float target, float k, float* energy, float grad[6], float hess[36]) {
  dgpu::float3 xs[2] = {{x[0], x[1], x[2]}, {x[3], x[4], x[5]}};
  dgpu::TermEvalF<2> te;
  dgpu::clearTerm(te);
  dgpu::evalSeamF(xs, target, k, te);
  *energy = te.energy;
  for (int a = 0; a < 2; ++a) {
    grad[3 * a] = te.grad[a].x;
    grad[3 * a + 1] = te.grad[a].y;
    grad[3 * a + 2] = te.grad[a].z;
    for (int b = 0; b < 2; ++b) storeMat(te.hess[a][b], hess + 9 * (2 * a + b));
  }
}

void ref_eval_friction(const float dx[3], const float n[3], float mu_lambda, float eps, float* energy, float grad[3],
                       float hess[9]) {
  dgpu::TermEvalF<1> te;
  dgpu::clearTerm(te);
  dgpu::evalFrictionF({dx[0], dx[1], dx[2]}, {n[0], n[1], n[2]}, mu_lambda, eps, te);
  *energy = te.energy;
  grad[0] = te.grad[0].x;
  grad[1] = te.grad[0].y;
  grad[2] = te.grad[0].z;
  storeMat(te.hess[0][0], hess);
}

float ref_field_sample(const drape_field_desc* f, const float p[3]) {
  return dgpu::fieldSample(f->values, fieldInfo(f), {p[0], p[1], p[2]});
}

void ref_field_gradient(const drape_field_desc* f, const float p[3], float g[3]) {
  const dgpu::float3 r = dgpu::fieldGradient(f->values, fieldInfo(f), {p[0], p[1], p[2]});
  g[0] = r.x;
  g[1] = r.y;
  g[2] = r.z;
}

void ref_collide_body(const drape_field_desc* f, float radius, float friction, const float x_prev[3], float x[3]) {
  dgpu::float3 xf{x[0], x[1], x[2]};
  dgpu::collideBodyF(f->values, fieldInfo(f), radius, friction, {x_prev[0], x_prev[1], x_prev[2]}, xf);
  x[0] = xf.x;
  x[1] = xf.y;
  x[2] = xf.z;
}

void ref_land_on_body(const drape_field_desc* f, float radius, const float from[3], const float to[3], float out[3]) {
  const dgpu::float3 r =
      dgpu::landOnBodyF(f->values, fieldInfo(f), radius, {from[0], from[1], from[2]}, {to[0], to[1], to[2]});
  out[0] = r.x;
  out[1] = r.y;
  out[2] = r.z;
}

int ref_invert_spd3(const float a[9], float out[9]) {
  const dgpu::Block3 b = blockFromRowMajor(a);
  bool ok = false;
  const dgpu::Mat3 inv = dgpu::invertSpd3(dgpu::loadBlock(b), ok);
  storeMat(inv, out);
  return ok ? 1 : 0;
}

/* The reference's two-level deterministic float reduction (k_reduce_partial + k_reduce_final). */
float ref_reduce(const float* data, uint32_t count) {
  Device d;
  const BufferId input = d.upload(std::vector<float>(data, data + count));
  const BufferId spec = d.upload(std::vector<dgpu::ReduceSpec>{{count, dgpu::kReduceRr, {0, 0}}});
  const BufferId partials = d.array<float>(count / dgpu::kReduceBlock + 1);
  const BufferId scalars = d.array<dgpu::CgScalars>(1);
  d.dev.begin();
  d.dispatch(Kernel::ReducePartial, count / dgpu::kReduceBlock + 1, {spec, input, partials});
  d.dispatch(Kernel::ReduceFinal, 1, {spec, partials, scalars});
  d.dev.submitAndWait();
  return d.view<dgpu::CgScalars>(scalars)->rr;
}

/* The reference's block-Jacobi PCG dispatch sequence (gpu_solver_core.cpp:312-368) on a given FP32 system: blocks
   are 9 floats per slot, row-major. */
int ref_pcg(uint32_t n, const uint32_t* row_start, const uint32_t* col_index, const float* blocks,
            const uint8_t* pinned, const uint8_t* active, const float* normals, const float* grad, int max_iterations,
            float tolerance, float* step, float* resid, int* iterations) {
  try {
    Device d;
    const uint32_t B = row_start[n];
    std::vector<dgpu::GpuParticle> parts(n);
    std::vector<uint32_t> diag(n);
    for (uint32_t i = 0; i < n; ++i) {
      parts[i] = {1.0f, 0, 0, pinned[i] ? 1u : 0u};
      diag[i] = B;
      for (uint32_t k = row_start[i]; k < row_start[i + 1]; ++k)
        if (col_index[k] == i) diag[i] = k;
      if (diag[i] == B) return -1;
    }
    std::vector<dgpu::Block3> bl(B);
    for (uint32_t k = 0; k < B; ++k) bl[k] = blockFromRowMajor(blocks + 9 * k);
    std::vector<dgpu::GpuContact> cs(n);
    std::vector<dgpu::float4> g(n);
    for (uint32_t i = 0; i < n; ++i) {
      cs[i].active = active && active[i] ? 1u : 0u;
      cs[i].nearBody = cs[i].active;
      if (normals) cs[i].normal = {normals[3 * i], normals[3 * i + 1], normals[3 * i + 2], 0.0f};
      g[i] = {grad[3 * i], grad[3 * i + 1], grad[3 * i + 2], 0.0f};
    }
    dgpu::StepParams sp{};
    sp.n = n;
    sp.nBlocks = B;
    sp.cgTolerance = tolerance;
    sp.maxCgIterations = static_cast<uint>(max_iterations);
    const BufferId params = d.upload(std::vector<dgpu::StepParams>{sp});
    const BufferId pinfo = d.upload(parts), rows = d.upload(std::vector<uint32_t>(row_start, row_start + n + 1)),
                   cols = d.upload(std::vector<uint32_t>(col_index, col_index + B)), dg = d.upload(diag),
                   blk = d.upload(bl), contact = d.upload(cs), gradB = d.upload(g);
    const BufferId scalars = d.array<dgpu::CgScalars>(1), partials = d.array<float>(n / 256 + 1);
    BufferId stepB = d.array<dgpu::float4>(n), r = d.array<dgpu::float4>(n), z = d.array<dgpu::float4>(n),
             p = d.array<dgpu::float4>(n), ap = d.array<dgpu::float4>(n), apFull = d.array<dgpu::float4>(n),
             residB = d.array<dgpu::float4>(n), precond = d.array<dgpu::Block3>(n);
    const BufferId prodA = d.array<float>(n), prodB = d.array<float>(n);
    auto spec = [&](uint selector) { return d.upload(std::vector<dgpu::ReduceSpec>{{n, selector, {0, 0}}}); };
    const BufferId specRz = spec(dgpu::kReduceRz), specR0 = spec(dgpu::kReduceR0), specPAp = spec(dgpu::kReducePAp),
                   specRr = spec(dgpu::kReduceRr), specRzNew = spec(dgpu::kReduceRzNew);
    auto reduce = [&](BufferId sp2, BufferId input) {
      d.dispatch(Kernel::ReducePartial, n / 256 + 1, {sp2, input, partials});
      d.dispatch(Kernel::ReduceFinal, 1, {sp2, partials, scalars});
    };
    d.dev.begin();
    d.dispatch(Kernel::Precondition, n, {params, pinfo, dg, blk, precond});
    d.dispatch(Kernel::CgInit, n, {params, contact, precond, gradB, stepB, residB, r, z, p, prodA, prodB});
    reduce(specRz, prodA);
    reduce(specR0, prodB);
    for (int it = 0; it < max_iterations; ++it) {
      d.dispatch(Kernel::Spmv, n, {params, pinfo, rows, cols, blk, contact, scalars, p, apFull, ap, prodA});
      reduce(specPAp, prodA);
      d.dispatch(Kernel::CgAlpha, 1, {scalars});
      d.dispatch(Kernel::CgUpdate, n, {params, scalars, p, ap, apFull, stepB, r, residB, prodB});
      reduce(specRr, prodB);
      d.dispatch(Kernel::CgCheck, 1, {params, scalars});
      d.dispatch(Kernel::CgPrecond, n, {params, contact, scalars, precond, r, z, prodA});
      reduce(specRzNew, prodA);
      d.dispatch(Kernel::CgBeta, 1, {scalars});
      d.dispatch(Kernel::CgDirection, n, {params, scalars, z, p});
    }
    d.dev.submitAndWait();
    const auto* st = d.view<dgpu::float4>(stepB);
    const auto* rs = d.view<dgpu::float4>(residB);
    for (uint32_t i = 0; i < n; ++i) {
      step[3 * i] = st[i].x;
      step[3 * i + 1] = st[i].y;
      step[3 * i + 2] = st[i].z;
      resid[3 * i] = rs[i].x;
      resid[3 * i + 1] = rs[i].y;
      resid[3 * i + 2] = rs[i].z;
    }
    *iterations = static_cast<int>(d.view<dgpu::CgScalars>(scalars)->iteration);
    return 0;
  } catch (const std::exception&) {
    return -3;
  }
}

}  // extern "C"
