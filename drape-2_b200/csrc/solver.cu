// Host driver of the CUDA cloth solver and its C ABI (include/drape_cuda.h).
//
// The driver plays the role of the reference's GpuSolverCore (libs/sim/src/gpu/gpu_solver_core.cpp:41-407): it owns
// the model (model.hpp), the device buffers and one CUDA stream, and issues per substep
//   k_begin, then per Newton iteration k_activate, k_terms, k_assemble, k_solve (cooperative), then k_finish, k_advance_clock.
// Unlike the reference driver there is no host round trip inside a substep: energies, slope, line search and the
// Newton stop test are decided on the device. The host waits once per step() (once per frame in the drape runner, with
// the frame's statistics) to read the work counters and the error status (the bounded grid barrier's timeout).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <thread>
#include <climits>
#include <cmath>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/drape_cuda.h"
#include "../../include/drape_precond.h"
#include "device_buffer.hpp"
#include "device_model.hpp"
#include "kernels.cuh"
#include "solver_kernels.cuh"
#include "learned.hpp"
#include "model.hpp"

using drape_b200::Model;

namespace {

using dbuf::check;
#define CK(x) check((x), #x)
using dbuf::CountTransfers;
using dbuf::DBuf;
using dbuf::HostPinned;

thread_local std::string g_lastError;

}  // namespace

// Largest slot count of any solve block's contiguous row range (the split the device's blockRange makes).
static uint32_t maxBlockSlots(const uint32_t* rowStart, uint32_t n, int grid) {
  const uint32_t per = (n + static_cast<uint32_t>(grid) - 1) / static_cast<uint32_t>(grid);
  uint32_t most = 0;
  for (int b = 0; b < grid; ++b) {
    const uint32_t r0 = std::min<uint32_t>(n, static_cast<uint32_t>(b) * per), r1 = std::min<uint32_t>(n, r0 + per);
    most = std::max(most, rowStart[r1] - rowStart[r0]);
  }
  return most;
}

// Padded slots of the sliced layout k_solve_rows stages for its largest block (the rows in warps of 32, each warp's
// rows padded to its longest unpinned row; pinned rows take no slots), or UINT32_MAX when a block has more rows than
// k_solve_rows has threads.
static uint32_t maxSlicedSlots(const uint32_t* rowStart, const uint8_t* pinned, uint32_t n, int grid) {
  const uint32_t per = (n + static_cast<uint32_t>(grid) - 1) / static_cast<uint32_t>(grid);
  if (per > static_cast<uint32_t>(dcu::kRowThreads)) return UINT32_MAX;
  uint32_t most = 0;
  for (int b = 0; b < grid; ++b) {
    const uint32_t r0 = std::min<uint32_t>(n, static_cast<uint32_t>(b) * per), r1 = std::min<uint32_t>(n, r0 + per);
    uint32_t total = 0;
    for (uint32_t w0 = r0; w0 < r1; w0 += 32) {
      uint32_t len = 0;
      for (uint32_t i = w0; i < std::min(r1, w0 + 32); ++i)
        if (!pinned[i]) len = std::max(len, rowStart[i + 1] - rowStart[i]);
      total += 32 * len;
    }
    most = std::max(most, total);
  }
  return most;
}

struct drape_solver {
  int device = 0;
  int numSMs = 0;
  cudaStream_t stream = nullptr;
  std::string error;
  Model m;
  bool built = false;
  int solveGrid = 0, pointGrid = 0, assembleGrid = 0, termsGrid = 0, statsGrid = 0;
  unsigned long long barrierLimitNs = 2000000000ull;  // 2 s
  int failAfter = -1;
  static constexpr int kFrameSlots = 32;  // most frames one advanceFrames call runs before its host wait
  uint32_t solveSmemCap = 0;       // block slots one solve block can keep in shared memory
  uint32_t rowsSmemCap = 0;        // padded slots one k_solve_rows block can keep in shared memory
  // Learned preconditioner: the solver's own copy of the network and its workspace on this solver's CSR.
  std::unique_ptr<net::Network> net;
  net::GraphHandle netGraph;
  bool learnedOn = false;
  int precondRefresh = 1;           // run the network on every precondRefresh-th Newton iteration
  int precondSwitch = 0;            // block-Jacobi iterations before the learned preconditioner takes over
  int pcgVariant = 0;               // block-Jacobi PCG form (drape_cuda_set_pcg_variant)
  uint64_t netNewtonCounter = 0;
  size_t solveSmemBytes = 0;       // dynamic shared memory of the solve launch for the built scene
  size_t rowsSmemBytes = 0;        // k_solve_rows's, when the built scene fits it (0: it does not)

  DBuf<dcu::Particle> particle;
  DBuf<dcu::Fabric> fabric;
  DBuf<dcu::Garment> garment;
  DBuf<dcu::Stretch> stretch;
  DBuf<dcu::Hinge> hinge;
  DBuf<dcu::Seam> seam;
  DBuf<uint32_t> rowStart, colIndex, diagSlot, incStart, incEntry, offSlot, offStart, offCode;
  DBuf<float> fieldValues, blocks;
  DBuf<float4> x, v, xStart, yRel, u, grad, step, r, z, p0, p1, ap, apFull, resid, fExt, pinPos, precond;
  DBuf<float4> pm0, pm1, pz;  // the pipelined PCG's extra vectors
  DBuf<float4> stretchDer, hingeDer;
  DBuf<dcu::Contact> contact;
  DBuf<double> partials, statsPartials;
  DBuf<dcu::Control> ctl;
  DBuf<dcu::StatsOut> statsOut;
  DBuf<unsigned int> statsDone;
  HostPinned<dcu::Control> hCtl;
  HostPinned<dcu::StatsOut> hStats;  // one slot per frame of a multi-frame advance
  DBuf<int> cgLog;
  dcu::Dev dev{};
  uint64_t h2dBytes = 0, d2hBytes = 0;

  // Kernel timing (drape_cuda_profile): event pairs recorded around launches, folded in after each synchronisation.
  struct Pending {
    cudaEvent_t a, b;
    int kind;
  };
  int profiling = 0;  // 0 off, 1 every kernel, 2 k_solve only
  std::vector<cudaEvent_t> eventPool;
  std::vector<Pending> pending;
  drape_profile prof{};

  cudaEvent_t takeEvent() {
    if (eventPool.empty()) {
      cudaEvent_t e;
      CK(cudaEventCreate(&e));
      return e;
    }
    cudaEvent_t e = eventPool.back();
    eventPool.pop_back();
    return e;
  }
  // Records a start event when profiling kernels of this kind (1: all kernels, 2: only k_solve, kind 3); returns it
  // (or nullptr).
  cudaEvent_t profStart(int kind) {
    if (profiling == 0 || (profiling == 2 && kind != 3)) return nullptr;
    cudaEvent_t a = takeEvent();
    CK(cudaEventRecord(a, stream));
    return a;
  }
  void profStop(cudaEvent_t a, int kind) {
    if (!a) return;
    cudaEvent_t b = takeEvent();
    CK(cudaEventRecord(b, stream));
    pending.push_back({a, b, kind});
  }
  // After the stream has been synchronised.
  void collectProfile() {
    for (const auto& p : pending) {
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, p.a, p.b));
      prof.launches[p.kind] += 1;
      prof.milliseconds[p.kind] += ms;
      eventPool.push_back(p.a);
      eventPool.push_back(p.b);
    }
    pending.clear();
  }

  // ---- setup ----

  explicit drape_solver(int dev_) : device(dev_) {
    int count = 0;
    CK(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) throw std::runtime_error("cuda: no device " + std::to_string(device));
    CK(cudaSetDevice(device));
    cudaDeviceProp prop{};
    CK(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) throw std::runtime_error(std::string("cuda: device ") + prop.name + " is not sm_100");
    if (!prop.cooperativeLaunch) throw std::runtime_error("cuda: device does not support cooperative launch");
    numSMs = prop.multiProcessorCount;
    CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    // The solve kernels keep their rows' matrix blocks in shared memory: as many slots as the opt-in limit leaves.
    const void* solveKernels[] = {reinterpret_cast<const void*>(dcu::k_solve<false, 0>),
                                  reinterpret_cast<const void*>(dcu::k_solve<false, 1>),
                                  reinterpret_cast<const void*>(dcu::k_solve<false, 2>),
                                  reinterpret_cast<const void*>(dcu::k_solve<true, 0>),
                                  reinterpret_cast<const void*>(dcu::k_pcg_only)};
    size_t staticSmem = 0;
    for (const void* k : solveKernels) {
      cudaFuncAttributes fa{};
      CK(cudaFuncGetAttributes(&fa, k));
      staticSmem = std::max(staticSmem, fa.sharedSizeBytes);
    }
    solveSmemCap = static_cast<uint32_t>((prop.sharedMemPerBlockOptin - staticSmem) / dcu::kSmemSlotBytes);
    const int dynMax = static_cast<int>(solveSmemCap * dcu::kSmemSlotBytes);
    for (const void* k : solveKernels) {
      CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, dynMax));
      int perSM = 0;
      CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k, dcu::kSolveThreads, dynMax));
      if (perSM < 1) throw std::runtime_error("cuda: the solve kernel does not fit on an SM");
    }
    {
      const void* rowKernels[] = {reinterpret_cast<const void*>(dcu::k_solve_rows),
                                  reinterpret_cast<const void*>(dcu::k_solve_rows_learned)};
      size_t rowsStatic = 0;
      for (const void* k : rowKernels) {
        cudaFuncAttributes fa{};
        CK(cudaFuncGetAttributes(&fa, k));
        rowsStatic = std::max(rowsStatic, fa.sharedSizeBytes);
      }
      rowsSmemCap = static_cast<uint32_t>((prop.sharedMemPerBlockOptin - rowsStatic) / dcu::kSmemSlotBytes);
      const int rowsMax = static_cast<int>(rowsSmemCap * dcu::kSmemSlotBytes);
      for (const void* k : rowKernels) {
        CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, rowsMax));
        int perSM = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k, dcu::kRowThreads, rowsMax));
        if (perSM < 1) throw std::runtime_error("cuda: the resident-row solve kernel does not fit on an SM");
      }
    }
    solveGrid = numSMs;  // one 1024-thread block per SM: fewest barrier arrivals
    pointGrid = numSMs * 8;
    statsGrid = numSMs * 2;
    hCtl.alloc();
    hStats.alloc(kFrameSlots);
    ctl.alloc(1);
    partials.alloc(2 * static_cast<size_t>(solveGrid) * dcu::kPartialStride);  // two halves, alternating
    statsPartials.alloc(static_cast<size_t>(statsGrid) * 8);
    statsOut.alloc(kFrameSlots);
    statsDone.alloc(1);
    cgLog.alloc(dcu::kCgLogCapacity);
  }

  ~drape_solver() {
    if (stream) {
      cudaSetDevice(device);
      cudaStreamSynchronize(stream);
      for (const auto& p : pending) {
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
      }
      for (auto e : eventPool) cudaEventDestroy(e);
      for (auto& g : frameGraphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
      cudaStreamDestroy(stream);
    }
  }

  void use() const { CK(cudaSetDevice(device)); }

  std::vector<dcu::Particle> particleData() const { return dmodel::particles(m); }
  std::vector<dcu::Fabric> fabricData() const { return dmodel::fabrics(m); }
  std::vector<dcu::Garment> garmentData() const { return dmodel::garments(m); }
  std::vector<dcu::Hinge> hingeData() const { return dmodel::hinges(m); }
  std::vector<dcu::Seam> seamData() const { return dmodel::seams(m); }

  void build(const drape_scene_desc& scene) {
    use();
    Model next = Model::build(scene, false);  // the field is uploaded from the scene's samples below
    built = false;
    m = std::move(next);
    const uint32_t n = static_cast<uint32_t>(m.x.size());
    const uint32_t B = static_cast<uint32_t>(m.colIndex.size());
    const uint32_t SP = (B + 31u) & ~31u;
    cudaStream_t s = stream;
    particle.upload(particleData(), s);
    fabric.upload(fabricData(), s);
    garment.upload(garmentData(), s);
    stretch.upload(dmodel::stretches(m), s);
    hinge.upload(hingeData(), s);
    seam.upload(seamData(), s);
    rowStart.upload(m.rowStart, s);
    colIndex.upload(dmodel::columns(m), s);
    diagSlot.upload(m.diagSlot, s);
    incStart.upload(m.incStart, s);
    incEntry.upload(m.incEntry, s);
    offSlot.upload(m.offSlot, s);
    offStart.upload(m.offStart, s);
    offCode.upload(m.offCode, s);
    if (m.fieldCount > 0) {
      fieldValues.upload(m.fieldData(), m.fieldCount, s);
      CK(cudaStreamSynchronize(s));  // the copy has read the caller's samples; the model keeps no pointer to them
      m.fieldSource = nullptr;
    } else {
      fieldValues.alloc(1);
    }
    blocks.alloc(static_cast<size_t>(SP) * 9);
    for (DBuf<float4>* b : {&x, &v, &xStart, &yRel, &u, &grad, &step, &r, &z, &p0, &p1, &ap, &apFull, &resid, &fExt, &pinPos,
                            &pm0, &pm1, &pz})
      b->alloc(n);
    precond.alloc(static_cast<size_t>(n) * 3);
    stretchDer.alloc(std::max<size_t>(1, 6 * m.stretch.size()));
    hingeDer.alloc(std::max<size_t>(1, 4 * m.hinges.size()));
    contact.alloc(n);
    {
      std::vector<float4> xs, vs, fe, pp;
      dmodel::state(m, xs, vs, fe, pp);
      x.upload(xs, s);
      v.upload(vs, s);
      fExt.upload(fe, s);
      pinPos.upload(pp, s);
    }
    dcu::Control c0{};
    CK(cudaMemcpyAsync(ctl.p, &c0, sizeof(c0), cudaMemcpyHostToDevice, s));
    // Launch view.
    dcu::Dev d{};
    dmodel::params(m, SP, barrierLimitNs, d);
    d.P.smemSlots = std::min(solveSmemCap, maxBlockSlots(m.rowStart.data(), n, solveGrid));
    solveSmemBytes = static_cast<size_t>(d.P.smemSlots) * dcu::kSmemSlotBytes;
    {
      const uint32_t sliced = maxSlicedSlots(m.rowStart.data(), m.pinned.data(), n, solveGrid);
      const bool fits = sliced <= rowsSmemCap;
      d.P.slicedSlots = fits ? std::max<uint32_t>(sliced, 1u) : 0u;
      rowsSmemBytes = fits ? static_cast<size_t>(d.P.slicedSlots) * dcu::kSmemSlotBytes : 0;
    }
    d.fieldValues = fieldValues.p;
    d.particle = particle.p;
    d.fabric = fabric.p;
    d.garment = garment.p;
    d.stretch = stretch.p;
    d.hinge = hinge.p;
    d.seam = seam.p;
    d.rowStart = rowStart.p;
    d.colIndex = colIndex.p;
    d.diagSlot = diagSlot.p;
    d.incStart = incStart.p;
    d.incEntry = incEntry.p;
    d.offSlot = offSlot.p;
    d.offStart = offStart.p;
    d.offCode = offCode.p;
    d.x = x.p;
    d.v = v.p;
    d.xStart = xStart.p;
    d.yRel = yRel.p;
    d.u = u.p;
    d.grad = grad.p;
    d.step = step.p;
    d.r = r.p;
    d.z = z.p;
    d.p0 = p0.p;
    d.p1 = p1.p;
    d.ap = ap.p;
    d.apFull = apFull.p;
    d.resid = resid.p;
    d.pm0 = pm0.p;
    d.pm1 = pm1.p;
    d.pz = pz.p;
    d.P.pcgVariant = pcgVariant;
    d.stretchDer = stretchDer.p;
    d.hingeDer = hingeDer.p;
    d.fExt = fExt.p;
    d.pinPos = pinPos.p;
    d.blocks = blocks.p;
    d.precond = precond.p;
    d.contact = contact.p;
    d.partials = partials.p;
    d.ctl = ctl.p;
    d.cgLog = cgLog.p;
    dev = d;
    netGraph.reset();
    if (learnedOn) bindNet();
    assembleGrid = static_cast<int>(std::max<uint32_t>(1, std::min<uint32_t>((B + dcu::kAssembleThreads - 1) / dcu::kAssembleThreads,
                                                                           static_cast<uint32_t>(numSMs) * 64)));
    const size_t terms = m.stretch.size() + m.hinges.size();
    termsGrid = static_cast<int>(std::max<size_t>(1, std::min<size_t>((terms + dcu::kTermThreads - 1) / dcu::kTermThreads,
                                                                      static_cast<size_t>(numSMs) * 16)));
    CK(cudaStreamSynchronize(s));
    built = true;
  }

  // The network's workspace on this solver's CSR; the learned factor and transposed-slot map go into the device view.
  void bindNet() {
    const uint32_t n = static_cast<uint32_t>(m.pinned.size()), B = static_cast<uint32_t>(m.colIndex.size());
    const std::vector<uint32_t> cols = dmodel::columns(m);
    netGraph = net->bind(n, B, dev.P.slotsPadded, m.rowStart.data(), cols.data(), rowStart.p, colIndex.p, blocks.p,
                         reinterpret_cast<const uint8_t*>(particle.p) + offsetof(dcu::Particle, pinned),
                         sizeof(dcu::Particle),
                         reinterpret_cast<const uint8_t*>(contact.p) + offsetof(dcu::Contact, active),
                         sizeof(dcu::Contact), stream, true);
    dev.Lf = net->graphOf(*netGraph).L;
    dev.tslot = net->graphOf(*netGraph).tslot;
    dev.LfRows = net->graphOf(*netGraph).LF;
    netNewtonCounter = 0;
  }

  void setPrecond(drape_precond* p) {
    if (!p) {
      learnedOn = false;
      netGraph.reset();
      dev.Lf = nullptr;
      dev.tslot = nullptr;
      dev.LfRows = nullptr;
      return;
    }
    if (!p->net) throw std::invalid_argument("null preconditioner handle");
    std::vector<float> w(net::Layout::kCount);
    p->net->getParams(w.data(), w.size());
    if (!net) net = std::make_unique<net::Network>(device);
    net->setParams(w.data(), w.size());
    learnedOn = true;
    if (built) bindNet();
  }

  void requireBuilt() const {
    if (!built) throw std::logic_error("not built");
  }

  // ---- model <-> device ----

  // Device -> model: positions, velocities and contact forces (the state the device advances).
  void syncToModel() {
    use();
    const size_t n = m.x.size();
    std::vector<float4> xs(n), vs(n);
    std::vector<dcu::Contact> cs(n);
    if (n) {
      CK(cudaMemcpyAsync(xs.data(), x.p, sizeof(float4) * n, cudaMemcpyDeviceToHost, stream));
      CK(cudaMemcpyAsync(vs.data(), v.p, sizeof(float4) * n, cudaMemcpyDeviceToHost, stream));
      CK(cudaMemcpyAsync(cs.data(), contact.p, sizeof(dcu::Contact) * n, cudaMemcpyDeviceToHost, stream));
      CK(cudaStreamSynchronize(stream));
      d2hBytes += (2 * sizeof(float4) + sizeof(dcu::Contact)) * n;
    }
    for (size_t i = 0; i < n; ++i) {
      m.x[i] = {xs[i].x, xs[i].y, xs[i].z};
      m.v[i] = {vs[i].x, vs[i].y, vs[i].z};
      m.contactForce[i] = cs[i].force;
    }
  }

  // Model -> device: everything the model may have changed (restore, setPhase, updateFabric).
  void syncFromModel() {
    use();
    const size_t n = m.x.size();
    std::vector<float4> xs(n), vs(n);
    std::vector<dcu::Contact> cs(n);
    if (n) {
      CK(cudaMemcpyAsync(cs.data(), contact.p, sizeof(dcu::Contact) * n, cudaMemcpyDeviceToHost, stream));
      CK(cudaStreamSynchronize(stream));
    }
    for (size_t i = 0; i < n; ++i) {
      xs[i] = dmodel::f4(m.x[i]);
      vs[i] = dmodel::f4(m.v[i]);
      cs[i].force = static_cast<float>(m.contactForce[i]);
    }
    x.upload(xs, stream);
    v.upload(vs, stream);
    contact.upload(cs, stream);
    particle.upload(particleData(), stream);
    fabric.upload(fabricData(), stream);
    garment.upload(garmentData(), stream);
    hinge.upload(hingeData(), stream);
    seam.upload(seamData(), stream);
    CK(cudaStreamSynchronize(stream));
  }

  // ---- stepping ----

  void resetControlAfterError() {
    dcu::Control c{};
    CK(cudaMemcpy(&c, ctl.p, sizeof(c), cudaMemcpyDeviceToHost));
    c.error = 0;
    c.barrierArrivals = 0;
    CK(cudaMemcpy(ctl.p, &c, sizeof(c), cudaMemcpyHostToDevice));
  }

  // The reference-order PCG runs over resident rows (k_solve_rows) where the built scene fits it; bit-identical to
  // k_solve<false, 0>, which variant 3 forces. The learned preconditioner runs over resident rows too
  // (k_solve_rows_learned) unless block-Jacobi iterations come first (precondSwitch) or variant 3 forces k_solve<true>.
  bool usesResidentRows(const dcu::Dev& d) const {
    return d.P.pcgVariant == 0 && rowsSmemBytes > 0 && (!(learnedOn && netGraph) || precondSwitch == 0);
  }

  void launchSolve(const dcu::Dev& d) {
    const bool rows = usesResidentRows(d);
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(solveGrid);
    cfg.blockDim = dim3(rows ? dcu::kRowThreads : dcu::kSolveThreads);
    cfg.dynamicSmemBytes = rows ? rowsSmemBytes : solveSmemBytes;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;  // co-resident blocks for the grid barrier; capturable in a graph
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (learnedOn && netGraph) {
      if (rows)
        CK(cudaLaunchKernelEx(&cfg, dcu::k_solve_rows_learned, d));
      else
        CK(cudaLaunchKernelEx(&cfg, dcu::k_solve<true, 0>, d));
    } else if (rows) {
      CK(cudaLaunchKernelEx(&cfg, dcu::k_solve_rows, d));
    } else if (d.P.pcgVariant == 1) {
      CK(cudaLaunchKernelEx(&cfg, dcu::k_solve<false, 1>, d));
    } else if (d.P.pcgVariant == 2) {
      CK(cudaLaunchKernelEx(&cfg, dcu::k_solve<false, 2>, d));
    } else {
      CK(cudaLaunchKernelEx(&cfg, dcu::k_solve<false, 0>, d));
    }
  }

  // Frame graphs: one frame's launches (its substeps, then the statistics into device slot f) captured once per slot and
  // replayed, one graph launch a frame instead of a dozen kernel launches. A graph is recaptured when the device view
  // or a launch parameter it was captured with changes; profiling and the learned preconditioner launch directly.
  struct FrameGraph {
    cudaGraphExec_t exec = nullptr;
    dcu::Dev dev{};
    double h = 0;
    int substeps = 0, iterations = 0, precondSwitch = 0;
    unsigned long long barrierLimitNs = 0;
  };
  FrameGraph frameGraphs[kFrameSlots];
  bool frameGraphsUsable = true;

  bool launchFrameGraph(double h, int substeps, int iterations, int slot) {
    if (!frameGraphsUsable || profiling != 0 || (learnedOn && netGraph)) return false;
    FrameGraph& g = frameGraphs[slot];
    if (!g.exec || g.h != h || g.substeps != substeps || g.iterations != iterations ||
        g.precondSwitch != precondSwitch || g.barrierLimitNs != barrierLimitNs ||
        std::memcmp(&g.dev, &dev, sizeof(dcu::Dev)) != 0) {
      if (g.exec) CK(cudaGraphExecDestroy(g.exec));
      g.exec = nullptr;
      const uint64_t bytes = d2hBytes;
      cudaGraph_t graph = nullptr;
      CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
      try {
        for (int k = 0; k < substeps; ++k) enqueueSubstep(h, iterations, false);
        enqueueStats(slot, false);
      } catch (...) {
        cudaStreamEndCapture(stream, &graph);
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        frameGraphsUsable = false;
        d2hBytes = bytes;
        return false;
      }
      d2hBytes = bytes;
      if (cudaStreamEndCapture(stream, &graph) != cudaSuccess || !graph ||
          cudaGraphInstantiate(&g.exec, graph, 0) != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        g.exec = nullptr;
        frameGraphsUsable = false;
        return false;
      }
      cudaGraphDestroy(graph);
      g.dev = dev;
      g.h = h;
      g.substeps = substeps;
      g.iterations = iterations;
      g.precondSwitch = precondSwitch;
      g.barrierLimitNs = barrierLimitNs;
    }
    CK(cudaGraphLaunch(g.exec, stream));
    for (int k = 0; k < substeps; ++k) advanceHostClock(h);
    return true;
  }

  // The host copy of the Assembling garments' clocks, which k_advance_clock advances on the device.
  void advanceHostClock(double h) {
    for (auto& g : m.garments)
      if (g.phase == DRAPE_PHASE_ASSEMBLING) g.assemblyTime += h;
  }

  void enqueueSubstep(double h, int iterations, bool hostClock = true) {
    dcu::Dev d = dev;
    d.P.h = static_cast<float>(h);
    d.P.invH2 = static_cast<float>(1.0 / (h * h));
    d.P.hD = h;
    d.P.barrierLimitNs = barrierLimitNs;
    d.P.learnedSwitch = precondSwitch;
    const uint32_t n = d.P.n;
    const int pg = std::max(1, static_cast<int>(std::min<uint32_t>((n + 255) / 256, static_cast<uint32_t>(pointGrid))));
    cudaEvent_t e = profStart(0);
    dcu::k_begin<<<pg, 256, 0, stream>>>(d);
    CK(cudaGetLastError());
    profStop(e, 0);
    for (int it = 0; it < iterations; ++it) {
      e = profStart(1);
      dcu::k_activate<<<pg, 256, 0, stream>>>(d);
      profStop(e, 1);
      e = profStart(2);
      dcu::k_terms<<<termsGrid, dcu::kTermThreads, 0, stream>>>(d);
      profStop(e, 2);
      e = profStart(2);
      dcu::k_assemble<<<assembleGrid, dcu::kAssembleThreads, 0, stream>>>(d);
      CK(cudaGetLastError());
      profStop(e, 2);
      if (learnedOn && netGraph && netNewtonCounter++ % static_cast<uint64_t>(precondRefresh) == 0) {
        e = profStart(6);
        net->forwardOn(net->graphOf(*netGraph), stream, false, &ctl.p->error);
        profStop(e, 6);
      }
      e = profStart(3);
      launchSolve(d);
      profStop(e, 3);
    }
    e = profStart(4);
    dcu::k_finish<<<pg, 256, 0, stream>>>(d);
    dcu::k_advance_clock<<<1, 32, 0, stream>>>(d);
    CK(cudaGetLastError());
    profStop(e, 4);
    if (hostClock) advanceHostClock(h);
  }

  // Waits for the stream by polling it: the per-frame waits of stepping and of the drape runner wake up without the
  // scheduling delay a blocking synchronise can take on a busy host.
  // Polls for up to waitSpinUs microseconds, then sleeps 20 us between polls: a drape's waits (one per batch of
  // frames, ~14 ms of device work) do not keep a host core busy, which a CPU-quota-limited host would throttle while
  // the device drains its queue. waitSpinUs = UINT32_MAX polls without sleeping.
  uint32_t waitSpinUs = 200;
  void waitStream() {
    const auto start = std::chrono::steady_clock::now();
    for (;;) {
      const cudaError_t e = cudaStreamQuery(stream);
      if (e == cudaSuccess) return;
      if (e != cudaErrorNotReady) CK(e);
      if (waitSpinUs != UINT32_MAX &&
          std::chrono::steady_clock::now() - start > std::chrono::microseconds(waitSpinUs))
        std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
  }

  void readControl() {
    CK(cudaMemcpyAsync(hCtl.p, ctl.p, sizeof(dcu::Control), cudaMemcpyDeviceToHost, stream));
    waitStream();
    d2hBytes += sizeof(dcu::Control);
    collectProfile();
    checkControl();
  }

  // After the control block has reached hCtl: a device error status becomes std::runtime_error("cuda: ...").
  void checkControl() {
    if (hCtl.p->error != 0) {
      const int e = hCtl.p->error;
      resetControlAfterError();
      throw std::runtime_error(e == 1 ? "cuda: a grid barrier timed out (the step was abandoned)"
                                      : "cuda: device error status " + std::to_string(e));
    }
  }

  void advance(double dt, int substeps, int iterations) {
    requireBuilt();
    use();
    if (failAfter == 0) throw std::runtime_error("cuda: injected device failure");
    if (failAfter > 0) --failAfter;
    if (m.x.empty()) return;
    const int sub = std::max(1, substeps);
    const double h = dt / sub;
    const int its = std::max(1, iterations);
    for (int k = 0; k < sub; ++k) enqueueSubstep(h, its);
    readControl();
  }

  // The statistics of the state after this frame into device slot `slot`; with `copy`, also to the host slot. A batch
  // of frames copies its slots once at its end (advanceFrames), so the stream carries one small device-to-host copy
  // per batch instead of one per frame.
  void enqueueStats(int slot = 0, bool copy = true) {
    cudaEvent_t e = profStart(5);
    dcu::k_stats<<<statsGrid, 256, 0, stream>>>(dev, statsPartials.p, statsDone.p, statsOut.p + slot);
    CK(cudaGetLastError());
    profStop(e, 5);
    if (copy) {
      CK(cudaMemcpyAsync(hStats.p + slot, statsOut.p + slot, sizeof(dcu::StatsOut), cudaMemcpyDeviceToHost, stream));
      d2hBytes += sizeof(dcu::StatsOut);
    }
  }

  drape_stats stats() {
    requireBuilt();
    use();
    if (m.x.empty()) return drape_stats{};
    enqueueStats();
    waitStream();
    collectProfile();
    return hostStats();
  }

  // `frames` frames, each followed by its statistics, with one host synchronisation at the end: out[f] is the state
  // after frame f. One frame is the drape runner's per-frame pair of calls (advance, stats); several let the runner
  // keep the device busy across frames and decide on their statistics afterwards.
  void advanceFrames(double dt, int substeps, int iterations, int frames, drape_stats* out) {
    requireBuilt();
    use();
    if (frames < 1 || frames > kFrameSlots) throw std::invalid_argument("frames per advance out of range");
    if (failAfter == 0) throw std::runtime_error("cuda: injected device failure");
    if (failAfter > 0) failAfter = std::max(0, failAfter - frames);
    if (m.x.empty()) {
      for (int f = 0; f < frames; ++f) out[f] = drape_stats{};
      return;
    }
    const int sub = std::max(1, substeps);
    const double h = dt / sub;
    const int its = std::max(1, iterations);
    for (int f = 0; f < frames; ++f) {
      if (launchFrameGraph(h, sub, its, f)) continue;
      for (int k = 0; k < sub; ++k) enqueueSubstep(h, its);
      enqueueStats(f, false);
    }
    CK(cudaMemcpyAsync(hStats.p, statsOut.p, sizeof(dcu::StatsOut) * frames, cudaMemcpyDeviceToHost, stream));
    d2hBytes += sizeof(dcu::StatsOut) * frames;
    CK(cudaMemcpyAsync(hCtl.p, ctl.p, sizeof(dcu::Control), cudaMemcpyDeviceToHost, stream));
    d2hBytes += sizeof(dcu::Control);
    waitStream();
    collectProfile();
    checkControl();
    for (int f = 0; f < frames; ++f) {
      out[f] = hostStats(f);
      if (frameTimes.size() < kFrameTimeCapacity) frameTimes.push_back({hStats.p[f].beginNs, hStats.p[f].endNs});
    }
  }

  // Device timestamps (%globaltimer, ns) of the frames run in batches since the last read: the frame's first kernel
  // and the end of its statistics. Consecutive frames show the device-side duration of each frame and the idle time
  // between frames.
  static constexpr size_t kFrameTimeCapacity = 1u << 16;
  std::vector<std::pair<unsigned long long, unsigned long long>> frameTimes;
  // Host seconds of the last drape_to_rest: [0] set-up (phase change, first snapshot), [1] the frame loop, [2] the
  // return (everything after the loop).
  double runnerHostSeconds[3] = {0.0, 0.0, 0.0};

  drape_stats advanceWithStats(double dt, int substeps, int iterations) {
    drape_stats st{};
    advanceFrames(dt, substeps, iterations, 1, &st);
    return st;
  }

  drape_stats hostStats(int slot = 0) const {
    drape_stats st{};
    const dcu::StatsOut& s = hStats.p[slot];
    st.has_non_finite = s.nonFinite;
    st.kinetic_energy = s.kineticEnergy;
    st.rms_speed = s.moving ? std::sqrt(s.sumV2 / static_cast<double>(s.moving)) : 0.0;
    st.max_seam_gap = s.maxSeamGap;
    st.max_body_penetration = m.hasBody ? s.maxPenetration : 0.0;
    return st;
  }

  drape_counters counters() {
    use();
    CK(cudaMemcpyAsync(hCtl.p, ctl.p, sizeof(dcu::Control), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    drape_counters c{};
    c.substeps = hCtl.p->substeps;
    c.newton_iterations = hCtl.p->newtonIterations;
    c.cg_iterations = hCtl.p->cgIterations;
    c.line_search_halvings = hCtl.p->lineSearchHalvings;
    c.precond_fallbacks = hCtl.p->precondFallbacks;
    c.learned_solves = hCtl.p->learnedSolves;
    c.pcg_nanoseconds = hCtl.p->pcgNs;
    return c;
  }

  void resetCounters() {
    use();
    CK(cudaMemcpyAsync(hCtl.p, ctl.p, sizeof(dcu::Control), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    dcu::Control c = *hCtl.p;
    c.substeps = c.newtonIterations = c.cgIterations = c.lineSearchHalvings = c.energyEvaluations = 0;
    c.learnedSolves = c.precondFallbacks = c.pcgNs = 0;
    *hCtl.p = c;
    CK(cudaMemcpyAsync(ctl.p, hCtl.p, sizeof(dcu::Control), cudaMemcpyHostToDevice, stream));
    CK(cudaStreamSynchronize(stream));
  }

  void readVec(const DBuf<float4>& b, float* out, size_t count) {
    requireBuilt();
    use();
    if (count != m.x.size()) throw std::invalid_argument("readPositions: span size must equal particleCount()");
    std::vector<float4> tmp(count);
    if (count) {
      CK(cudaMemcpyAsync(tmp.data(), b.p, sizeof(float4) * count, cudaMemcpyDeviceToHost, stream));
      CK(cudaStreamSynchronize(stream));
      d2hBytes += sizeof(float4) * count;
    }
    for (size_t i = 0; i < count; ++i) {
      out[3 * i] = tmp[i].x;
      out[3 * i + 1] = tmp[i].y;
      out[3 * i + 2] = tmp[i].z;
    }
  }

  // ---- device-side snapshots for the drape runner ----

  struct DeviceSnapshot {
    DBuf<float4> x, v;
    DBuf<dcu::Contact> contact;
    std::vector<int> phases;
    std::vector<double> assemblyTime;
    std::vector<float> seamStartGap;
  };
  // The drape runner's snapshots (the retry snapshot and a batch's start), kept across drapes so that a drape
  // allocates and frees no device memory (cudaFree synchronises the device, and either call can stall the host).
  DeviceSnapshot runnerSaved, runnerBatchStart;

  void saveTo(DeviceSnapshot& s) {
    const size_t n = m.x.size();
    if (s.x.n != n) {
      s.x.alloc(n);
      s.v.alloc(n);
      s.contact.alloc(n);
    }
    if (n) {
      CK(cudaMemcpyAsync(s.x.p, x.p, sizeof(float4) * n, cudaMemcpyDeviceToDevice, stream));
      CK(cudaMemcpyAsync(s.v.p, v.p, sizeof(float4) * n, cudaMemcpyDeviceToDevice, stream));
      CK(cudaMemcpyAsync(s.contact.p, contact.p, sizeof(dcu::Contact) * n, cudaMemcpyDeviceToDevice, stream));
    }
    s.phases.clear();
    s.assemblyTime.clear();
    for (const auto& g : m.garments) {
      s.phases.push_back(g.phase);
      s.assemblyTime.push_back(g.assemblyTime);
    }
    s.seamStartGap.clear();
    for (const auto& sp : m.seams) s.seamStartGap.push_back(sp.startGap);
  }

  void restoreFrom(const DeviceSnapshot& s) {
    const size_t n = m.x.size();
    if (n) {
      CK(cudaMemcpyAsync(x.p, s.x.p, sizeof(float4) * n, cudaMemcpyDeviceToDevice, stream));
      CK(cudaMemcpyAsync(v.p, s.v.p, sizeof(float4) * n, cudaMemcpyDeviceToDevice, stream));
      CK(cudaMemcpyAsync(contact.p, s.contact.p, sizeof(dcu::Contact) * n, cudaMemcpyDeviceToDevice, stream));
    }
    for (size_t g = 0; g < m.garments.size(); ++g) {
      m.garments[g].phase = s.phases[g];
      m.garments[g].assemblyTime = s.assemblyTime[g];
    }
    for (size_t k = 0; k < m.seams.size(); ++k) m.seams[k].startGap = s.seamStartGap[k];
    garment.upload(garmentData(), stream);
    seam.upload(seamData(), stream);
    CK(cudaStreamSynchronize(stream));
  }

  // Phase change without a full host round trip. Model::setPhase reads positions (the seams' start gaps) and writes
  // only the garment's phase and assembly time and its seams' start gaps, so Assembling downloads the positions and
  // uploads the garment and seam tables; nothing else of the model changes.
  void setPhase(const std::string& id, int phase) {
    requireBuilt();
    if (phase == DRAPE_PHASE_ASSEMBLING) {
      use();
      const size_t n = m.x.size();
      std::vector<float4> xs(n);
      if (n) {
        CK(cudaMemcpyAsync(xs.data(), x.p, sizeof(float4) * n, cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        d2hBytes += sizeof(float4) * n;
      }
      for (size_t i = 0; i < n; ++i) m.x[i] = {xs[i].x, xs[i].y, xs[i].z};
      m.setPhase(id, phase);
      garment.upload(garmentData(), stream);
      seam.upload(seamData(), stream);
      CK(cudaStreamSynchronize(stream));
    } else {
      m.setPhase(id, phase);
      use();
      garment.upload(garmentData(), stream);
      CK(cudaStreamSynchronize(stream));
    }
  }
};

// ---------------------------------------------------------------------------------------------------------------
// The drape runner (DrapeSession, libs/sim/src/drape_session.cpp:12-95) over the device solver, with its snapshots
// kept in device memory.

namespace {

constexpr double kTimeEps = 1e-9;

drape_drape_options defaultOptions() {
  drape_drape_options o{};
  o.substeps = 1;
  o.iterations = 2;
  o.frame_dt = 1.0 / 60.0;
  o.max_assembly_seconds = 3.0;
  o.seam_gap_done = 0.001;
  o.settle_rms_speed = 0.002;
  o.settle_hold_frames = 60;
  o.max_sim_seconds = 20.0;
  o.snapshot_every = 30;
  o.max_retries = 3;
  o.energy_rise_frames = 60;
  o.frames_per_wait = 10;
  return o;
}

drape_drape_result drapeToRest(drape_solver& s, const std::vector<std::string>& garments, const drape_drape_options& o) {
  drape_drape_result result{};
  auto setAll = [&](int phase) {
    for (const auto& g : garments) s.setPhase(g, phase);
  };
  const auto tStart = std::chrono::steady_clock::now();
  setAll(DRAPE_PHASE_ASSEMBLING);
  struct Saved {
    drape_solver::DeviceSnapshot& snap;
    double time = 0;
    int phase = DRAPE_PHASE_ASSEMBLING;
    double phaseTime = 0;
  } saved{s.runnerSaved};
  s.saveTo(saved.snap);
  const auto tLoop = std::chrono::steady_clock::now();
  int state = DRAPE_STATE_ASSEMBLING, phase = DRAPE_PHASE_ASSEMBLING;
  double time = 0, phaseTime = 0, lastEnergy = INFINITY;
  int substeps = o.substeps, stillFrames = 0, riseFrames = 0, keptFrames = 0;
  auto resetCounters = [&] {
    stillFrames = 0;
    riseFrames = 0;
    lastEnergy = INFINITY;
  };
  auto finished = [&] {
    return state == DRAPE_STATE_SETTLED || state == DRAPE_STATE_FAILED || state == DRAPE_STATE_TIMED_OUT;
  };
  // Frames run in batches of up to frames_per_wait with one host wait each. A batch ends where a decision is known in
  // advance to fall (the next snapshot frame, the time limits, the first frame that can complete the settle hold), so
  // those decisions land on its last frame. A decision that cannot be foreseen (the seam gap closing, a failure) on an
  // earlier frame j discards the batch's later frames: the state after frame j is rebuilt by restoring the batch's
  // start and replaying its first j + 1 frames, which the deterministic step reproduces bit for bit. The outcome is
  // the one-frame-per-wait runner's, frame for frame. The learned preconditioner refreshes on a Newton-iteration
  // count, which a replay would shift, so it keeps one frame per wait.
  const int perWait = s.learnedOn ? 1 : std::clamp(o.frames_per_wait, 1, drape_solver::kFrameSlots);
  drape_solver::DeviceSnapshot& batchStart = s.runnerBatchStart;
  drape_stats frameStats[drape_solver::kFrameSlots], replayStats[drape_solver::kFrameSlots];
  // The last two frames' seam gaps while Assembling: a batch stops at the frame where their trend meets
  // seam_gap_done, so the phase change seldom needs a replay.
  double gapPrev = NAN, gapLast = NAN;
  auto framesInBatch = [&] {
    const int settleIn = phase == DRAPE_PHASE_SETTLING ? std::max(1, o.settle_hold_frames - stillFrames) : INT_MAX;
    int gapIn = INT_MAX;
    if (phase == DRAPE_PHASE_ASSEMBLING && gapPrev > gapLast && gapLast >= o.seam_gap_done)
      gapIn = static_cast<int>(std::min(1e6, std::max(1.0, std::ceil((gapLast - o.seam_gap_done) / (gapPrev - gapLast)))));
    double t = time, pt = phaseTime;
    int k = 0, kept = keptFrames;
    for (;;) {
      ++k;
      ++kept;
      t += o.frame_dt;
      pt += o.frame_dt;
      if (k >= perWait || kept % o.snapshot_every == 0 || t >= o.max_sim_seconds - kTimeEps || k >= settleIn || k >= gapIn ||
          (phase == DRAPE_PHASE_ASSEMBLING && pt >= o.max_assembly_seconds - kTimeEps))
        break;
    }
    return s.failAfter > 0 ? std::min(k, s.failAfter) : k;
  };
  // Makes frame j the batch's last: the device state becomes the one after frame j.
  auto endBatchAt = [&](int j, int& k) {
    if (j + 1 >= k) return;
    s.restoreFrom(batchStart);
    const int injected = s.failAfter;
    s.failAfter = -1;
    s.advanceFrames(o.frame_dt, substeps, o.iterations, j + 1, replayStats);
    s.failAfter = injected;
    k = j + 1;
  };
  while (!finished()) {
    if (time >= o.max_sim_seconds - kTimeEps) {
      result.simulated_seconds = time;
      state = DRAPE_STATE_TIMED_OUT;
      break;
    }
    int k = framesInBatch();
    if (k > 1) s.saveTo(batchStart);
    s.advanceFrames(o.frame_dt, substeps, o.iterations, k, frameStats);
    for (int j = 0; j < k && !finished(); ++j) {
      const drape_stats& st = frameStats[j];
      ++result.frames_run;
      ++keptFrames;
      time += o.frame_dt;
      phaseTime += o.frame_dt;
      riseFrames = st.kinetic_energy > lastEnergy ? riseFrames + 1 : 0;
      lastEnergy = st.kinetic_energy;
      if (st.has_non_finite || riseFrames >= o.energy_rise_frames) {
        ++result.retries;
        if (result.retries > o.max_retries) {
          endBatchAt(j, k);
          result.retries = o.max_retries;
          result.failed = 1;
          result.simulated_seconds = time;
          state = DRAPE_STATE_FAILED;
          break;
        }
        s.restoreFrom(saved.snap);
        time = saved.time;
        phase = saved.phase;
        phaseTime = saved.phaseTime;
        keptFrames = static_cast<int>(saved.time / o.frame_dt + 0.5);
        substeps *= 2;
        resetCounters();
        gapPrev = gapLast = NAN;
        state = phase == DRAPE_PHASE_ASSEMBLING ? DRAPE_STATE_ASSEMBLING : DRAPE_STATE_SETTLING;
        break;
      }
      if (phase == DRAPE_PHASE_ASSEMBLING) {
        gapPrev = gapLast;
        gapLast = st.max_seam_gap;
        if (st.max_seam_gap < o.seam_gap_done || phaseTime >= o.max_assembly_seconds - kTimeEps) {
          endBatchAt(j, k);
          result.assembly_end_seam_gap = st.max_seam_gap;
          result.assembly_seconds = time;
          phase = DRAPE_PHASE_SETTLING;
          setAll(phase);
          phaseTime = 0;
          resetCounters();
        }
      } else {
        stillFrames = st.rms_speed < o.settle_rms_speed ? stillFrames + 1 : 0;
        if (stillFrames >= o.settle_hold_frames) {
          endBatchAt(j, k);
          result.settled = 1;
          result.simulated_seconds = time;
          state = DRAPE_STATE_SETTLED;
          break;
        }
      }
      if (keptFrames % o.snapshot_every == 0) {
        endBatchAt(j, k);
        s.saveTo(saved.snap);
        saved.time = time;
        saved.phase = phase;
        saved.phaseTime = phaseTime;
      }
      if (time >= o.max_sim_seconds - kTimeEps) {
        endBatchAt(j, k);
        result.simulated_seconds = time;
        state = DRAPE_STATE_TIMED_OUT;
        break;
      }
      state = phase == DRAPE_PHASE_ASSEMBLING ? DRAPE_STATE_ASSEMBLING : DRAPE_STATE_SETTLING;
    }
  }
  const auto tEnd = std::chrono::steady_clock::now();
  s.runnerHostSeconds[0] = std::chrono::duration<double>(tLoop - tStart).count();
  s.runnerHostSeconds[1] = std::chrono::duration<double>(tEnd - tLoop).count();
  return result;
}

template <class F>
int guarded(const drape_solver* cs, F&& f) {
  auto* s = const_cast<drape_solver*>(cs);
  CountTransfers count(s ? &s->h2dBytes : nullptr);
  try {
    f();
    return DRAPE_OK;
  } catch (const std::invalid_argument& e) {
    (s ? s->error : g_lastError) = e.what();
    return DRAPE_INVALID;
  } catch (const std::out_of_range& e) {
    (s ? s->error : g_lastError) = e.what();
    return DRAPE_OUT_OF_RANGE;
  } catch (const std::logic_error& e) {
    (s ? s->error : g_lastError) = e.what();
    return DRAPE_NOT_BUILT;
  } catch (const std::exception& e) {
    (s ? s->error : g_lastError) = e.what();
    return DRAPE_DEVICE_ERROR;
  }
}

void need(const drape_solver* s) {
  if (!s) throw std::invalid_argument("null solver handle");
}

void copyStructure(const Model& m, uint32_t* row_start, uint32_t* col_index, uint32_t* diag_slot,
                   uint32_t* stretch_slots, uint32_t* hinge_slots, uint32_t* seam_slots, uint32_t* stretch_v,
                   uint32_t* hinge_v, uint32_t* seam_ab) {
  if (row_start) std::copy(m.rowStart.begin(), m.rowStart.end(), row_start);
  if (col_index) std::copy(m.colIndex.begin(), m.colIndex.end(), col_index);
  if (diag_slot) std::copy(m.diagSlot.begin(), m.diagSlot.end(), diag_slot);
  for (size_t t = 0; t < m.stretch.size(); ++t) {
    if (stretch_slots) std::copy(m.stretchSlots[t].begin(), m.stretchSlots[t].end(), stretch_slots + 9 * t);
    if (stretch_v) std::copy(m.stretch[t].v.begin(), m.stretch[t].v.end(), stretch_v + 3 * t);
  }
  for (size_t h = 0; h < m.hinges.size(); ++h) {
    if (hinge_slots) std::copy(m.hingeSlots[h].begin(), m.hingeSlots[h].end(), hinge_slots + 16 * h);
    if (hinge_v) std::copy(m.hinges[h].v.begin(), m.hinges[h].v.end(), hinge_v + 4 * h);
  }
  for (size_t k = 0; k < m.seams.size(); ++k) {
    if (seam_slots) std::copy(m.seamSlots[k].begin(), m.seamSlots[k].end(), seam_slots + 4 * k);
    if (seam_ab) {
      seam_ab[2 * k] = m.seams[k].a;
      seam_ab[2 * k + 1] = m.seams[k].b;
    }
  }
}

}  // namespace

extern "C" {

int drape_cuda_version(void) { return 100; }

int drape_cuda_is_available(void) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return 0;
  }
  for (int d = 0; d < count; ++d) {
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, d) == cudaSuccess && prop.major == 10) {
      cudaFuncAttributes attr{};
      if (cudaFuncGetAttributes(&attr, dcu::k_solve<false, 0>) == cudaSuccess) return 1;
      cudaGetLastError();
    }
  }
  return 0;
}

int drape_cuda_create(int device, drape_solver** out) {
  return guarded(nullptr, [&] {
    if (!out) throw std::invalid_argument("null output pointer");
    *out = nullptr;
    *out = new drape_solver(device);
  });
}

void drape_cuda_destroy(drape_solver* s) { delete s; }

const char* drape_cuda_last_error(const drape_solver* s) { return s ? s->error.c_str() : g_lastError.c_str(); }

int drape_cuda_build(drape_solver* s, const drape_scene_desc* scene) {
  return guarded(s, [&] {
    need(s);
    if (!scene) throw std::invalid_argument("null scene");
    s->build(*scene);
  });
}

int drape_cuda_update_fabric(drape_solver* s, const char* garment, const drape_fabric* piece_fabric, uint32_t count) {
  return guarded(s, [&] {
    need(s);
    s->requireBuilt();
    s->syncToModel();
    s->m.updateFabric(garment ? garment : "", piece_fabric, count);
    s->syncFromModel();
  });
}

int drape_cuda_set_phase(drape_solver* s, const char* garment, int phase) {
  return guarded(s, [&] {
    need(s);
    if (phase != DRAPE_PHASE_ASSEMBLING && phase != DRAPE_PHASE_SETTLING) throw std::invalid_argument("unknown phase");
    s->setPhase(garment ? garment : "", phase);
  });
}

int drape_cuda_step(drape_solver* s, double dt, int substeps, int iterations) {
  return guarded(s, [&] {
    need(s);
    s->advance(dt, substeps, iterations);
  });
}

int drape_cuda_read_positions(const drape_solver* s, float* out, size_t count) {
  return guarded(s, [&] {
    need(s);
    const_cast<drape_solver*>(s)->readVec(s->x, out, count);
  });
}

int drape_cuda_read_velocities(const drape_solver* s, float* out, size_t count) {
  return guarded(s, [&] {
    need(s);
    const_cast<drape_solver*>(s)->readVec(s->v, out, count);
  });
}

int drape_cuda_stats(drape_solver* s, drape_stats* out) {
  return guarded(s, [&] {
    need(s);
    *out = s->stats();
  });
}

int drape_cuda_snapshot_sizes(const drape_solver* s, uint32_t* particles, uint32_t* garments, uint32_t* seams) {
  return guarded(s, [&] {
    need(s);
    s->requireBuilt();
    *particles = static_cast<uint32_t>(s->m.x.size());
    *garments = static_cast<uint32_t>(s->m.garments.size());
    *seams = static_cast<uint32_t>(s->m.seams.size());
  });
}

int drape_cuda_snapshot(const drape_solver* cs, float* positions, float* velocities, int32_t* phases,
                        double* assembly_time, float* seam_start_gap, double* contact_force) {
  return guarded(cs, [&] {
    need(cs);
    auto* s = const_cast<drape_solver*>(cs);
    s->requireBuilt();
    s->syncToModel();
    const auto& m = s->m;
    for (size_t i = 0; i < m.x.size(); ++i) {
      positions[3 * i] = m.x[i].x;
      positions[3 * i + 1] = m.x[i].y;
      positions[3 * i + 2] = m.x[i].z;
      velocities[3 * i] = m.v[i].x;
      velocities[3 * i + 1] = m.v[i].y;
      velocities[3 * i + 2] = m.v[i].z;
      contact_force[i] = m.contactForce[i];
    }
    for (size_t g = 0; g < m.garments.size(); ++g) {
      phases[g] = m.garments[g].phase;
      assembly_time[g] = m.garments[g].assemblyTime;
    }
    for (size_t k = 0; k < m.seams.size(); ++k) seam_start_gap[k] = m.seams[k].startGap;
  });
}

int drape_cuda_restore(drape_solver* s, const float* positions, const float* velocities, uint32_t particles,
                       const int32_t* phases, const double* assembly_time, uint32_t garments,
                       const float* seam_start_gap, uint32_t seams, const double* contact_force,
                       uint32_t contact_count) {
  return guarded(s, [&] {
    need(s);
    s->requireBuilt();
    auto& m = s->m;
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
      m.garments[g].phase = phases[g] == 0 ? DRAPE_PHASE_ASSEMBLING : DRAPE_PHASE_SETTLING;
      m.garments[g].assemblyTime = assembly_time[g];
    }
    if (seams == m.seams.size())
      for (size_t k = 0; k < seams; ++k) m.seams[k].startGap = seam_start_gap[k];
    s->syncFromModel();
  });
}

int drape_cuda_range(const drape_solver* s, const char* garment, uint32_t* offset, uint32_t* count) {
  return guarded(s, [&] {
    need(s);
    s->requireBuilt();
    const auto& g = s->m.garments[s->m.garmentIndex(garment ? garment : "")];
    *offset = g.offset;
    *count = g.count;
  });
}

int drape_cuda_particle_count(const drape_solver* s, size_t* out) {
  return guarded(s, [&] {
    need(s);
    *out = s->built ? s->m.x.size() : 0;
  });
}

int drape_cuda_drape_to_rest(drape_solver* s, const char* const* garments, uint32_t garment_count,
                             const drape_drape_options* options, drape_drape_result* out) {
  return guarded(s, [&] {
    need(s);
    s->requireBuilt();
    std::vector<std::string> ids;
    for (uint32_t k = 0; k < garment_count; ++k) ids.emplace_back(garments[k] ? garments[k] : "");
    for (const auto& id : ids) s->m.garmentIndex(id);
    const drape_drape_options o = options ? *options : defaultOptions();
    if (!(o.frame_dt > 0) || o.snapshot_every < 1 || o.substeps < 1)
      throw std::invalid_argument("frame_dt, substeps and snapshot_every must be positive");
    const auto t0 = std::chrono::steady_clock::now();
    *out = drapeToRest(*s, ids, o);
    s->runnerHostSeconds[2] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() -
                              s->runnerHostSeconds[0] - s->runnerHostSeconds[1];
  });
}

int drape_cuda_runner_host_seconds(const drape_solver* s, double* out) {
  return guarded(nullptr, [&] {
    if (!s || !out) throw std::invalid_argument("null argument");
    for (int k = 0; k < 3; ++k) out[k] = s->runnerHostSeconds[k];
  });
}

int drape_cuda_counters(const drape_solver* s, drape_counters* out) {
  return guarded(s, [&] {
    need(s);
    *out = const_cast<drape_solver*>(s)->counters();
  });
}

int drape_cuda_reset_counters(drape_solver* s) {
  return guarded(s, [&] {
    need(s);
    s->resetCounters();
  });
}

int drape_cuda_cg_history(const drape_solver* cs, int32_t* out, size_t capacity, size_t* count) {
  return guarded(cs, [&] {
    need(cs);
    auto* s = const_cast<drape_solver*>(cs);
    const drape_counters c = s->counters();
    const size_t total = static_cast<size_t>(c.newton_iterations);
    const size_t kept = std::min<size_t>(total, dcu::kCgLogCapacity);
    const size_t take = std::min(kept, capacity);
    std::vector<int> all(dcu::kCgLogCapacity);
    CK(cudaMemcpy(all.data(), s->cgLog.p, sizeof(int) * all.size(), cudaMemcpyDeviceToHost));
    const size_t first = total - kept;  // oldest kept index
    for (size_t k = 0; k < take; ++k) out[k] = all[(first + k) % dcu::kCgLogCapacity];
    *count = take;
  });
}

int drape_cuda_stream(const drape_solver* s, void** stream) {
  return guarded(s, [&] {
    need(s);
    *stream = static_cast<void*>(s->stream);
  });
}

int drape_cuda_profile(drape_solver* s, int enable) {
  return guarded(s, [&] {
    need(s);
    s->use();
    CK(cudaStreamSynchronize(s->stream));
    s->collectProfile();
    s->profiling = enable == 2 ? 2 : (enable != 0 ? 1 : 0);
    if (s->profiling) {
      s->prof = drape_profile{};
      const drape_counters c = s->counters();
      s->prof.cg_iterations = -c.cg_iterations;  // made relative in drape_cuda_profile_read
      s->prof.energy_evaluations = -s->hCtl.p->energyEvaluations;
    }
  });
}

int drape_cuda_profile_read(const drape_solver* cs, drape_profile* out) {
  return guarded(cs, [&] {
    need(cs);
    auto* s = const_cast<drape_solver*>(cs);
    s->use();
    CK(cudaStreamSynchronize(s->stream));
    s->collectProfile();
    const drape_counters c = s->counters();
    *out = s->prof;
    out->cg_iterations += c.cg_iterations;
    out->energy_evaluations += s->hCtl.p->energyEvaluations;
  });
}

int drape_cuda_transfer_bytes(const drape_solver* s, uint64_t* h2d, uint64_t* d2h) {
  return guarded(s, [&] {
    need(s);
    *h2d = s->h2dBytes;
    *d2h = s->d2hBytes;
  });
}

int drape_cuda_structure_sizes(const drape_solver* s, uint32_t sizes[5]) {
  return guarded(s, [&] {
    need(s);
    s->requireBuilt();
    sizes[0] = static_cast<uint32_t>(s->m.x.size());
    sizes[1] = static_cast<uint32_t>(s->m.colIndex.size());
    sizes[2] = static_cast<uint32_t>(s->m.stretch.size());
    sizes[3] = static_cast<uint32_t>(s->m.hinges.size());
    sizes[4] = static_cast<uint32_t>(s->m.seams.size());
  });
}

int drape_cuda_structure(const drape_solver* s, uint32_t* row_start, uint32_t* col_index, uint32_t* diag_slot,
                         uint32_t* stretch_slots, uint32_t* hinge_slots, uint32_t* seam_slots, uint32_t* stretch_v,
                         uint32_t* hinge_v, uint32_t* seam_ab) {
  return guarded(s, [&] {
    need(s);
    s->requireBuilt();
    copyStructure(s->m, row_start, col_index, diag_slot, stretch_slots, hinge_slots, seam_slots, stretch_v, hinge_v,
                  seam_ab);
  });
}

struct drape_model {
  Model m;
};

int drape_model_build(const drape_scene_desc* scene, drape_model** out) {
  return guarded(nullptr, [&] {
    if (!scene || !out) throw std::invalid_argument("null argument");
    *out = nullptr;
    auto* dm = new drape_model;
    try {
      dm->m = Model::build(*scene);
    } catch (...) {
      delete dm;
      throw;
    }
    *out = dm;
  });
}

void drape_model_destroy(drape_model* m) { delete m; }

const char* drape_model_last_error(void) { return g_lastError.c_str(); }

int drape_model_structure_sizes(const drape_model* dm, uint32_t sizes[5]) {
  return guarded(nullptr, [&] {
    if (!dm) throw std::invalid_argument("null model");
    sizes[0] = static_cast<uint32_t>(dm->m.x.size());
    sizes[1] = static_cast<uint32_t>(dm->m.colIndex.size());
    sizes[2] = static_cast<uint32_t>(dm->m.stretch.size());
    sizes[3] = static_cast<uint32_t>(dm->m.hinges.size());
    sizes[4] = static_cast<uint32_t>(dm->m.seams.size());
  });
}

int drape_model_structure(const drape_model* dm, uint32_t* row_start, uint32_t* col_index, uint32_t* diag_slot,
                          uint32_t* stretch_slots, uint32_t* hinge_slots, uint32_t* seam_slots, uint32_t* stretch_v,
                          uint32_t* hinge_v, uint32_t* seam_ab) {
  return guarded(nullptr, [&] {
    if (!dm) throw std::invalid_argument("null model");
    copyStructure(dm->m, row_start, col_index, diag_slot, stretch_slots, hinge_slots, seam_slots, stretch_v, hinge_v,
                  seam_ab);
  });
}

int drape_model_gather_sizes(const drape_model* dm, uint32_t sizes[4]) {
  return guarded(nullptr, [&] {
    if (!dm || !sizes) throw std::invalid_argument("null model or sizes");
    const Model& m = dm->m;
    sizes[0] = static_cast<uint32_t>(m.x.size());
    sizes[1] = static_cast<uint32_t>(m.incEntry.size());
    sizes[2] = static_cast<uint32_t>(m.offSlot.size());
    sizes[3] = static_cast<uint32_t>(m.offContrib.size());
  });
}

int drape_model_gather_lists(const drape_model* dm, uint32_t* inc_start, uint32_t* inc_entry, uint32_t* off_slot,
                             uint32_t* off_start, uint32_t* off_contrib) {
  return guarded(nullptr, [&] {
    if (!dm) throw std::invalid_argument("null model");
    const Model& m = dm->m;
    if (inc_start) std::copy(m.incStart.begin(), m.incStart.end(), inc_start);
    if (inc_entry) std::copy(m.incEntry.begin(), m.incEntry.end(), inc_entry);
    if (off_slot) std::copy(m.offSlot.begin(), m.offSlot.end(), off_slot);
    if (off_start) std::copy(m.offStart.begin(), m.offStart.end(), off_start);
    if (off_contrib) std::copy(m.offContrib.begin(), m.offContrib.end(), off_contrib);
  });
}

int drape_cuda_contact_candidates(drape_solver* s, const float* x_start, uint8_t* near_flag, float* normal,
                                  float* offset) {
  return guarded(s, [&] {
    need(s);
    s->requireBuilt();
    s->use();
    const size_t n = s->m.x.size();
    if (!n) return;
    std::vector<float4> xs(n);
    for (size_t i = 0; i < n; ++i) xs[i] = make_float4(x_start[3 * i], x_start[3 * i + 1], x_start[3 * i + 2], 0.0f);
    DBuf<float4> dx;
    DBuf<dcu::Contact> dc;
    dx.upload(xs, s->stream);
    dc.alloc(n);
    dcu::k_contact_candidates<<<std::max<int>(1, static_cast<int>((n + 255) / 256)), 256, 0, s->stream>>>(s->dev, dx.p, dc.p);
    CK(cudaGetLastError());
    std::vector<dcu::Contact> cs(n);
    CK(cudaMemcpyAsync(cs.data(), dc.p, sizeof(dcu::Contact) * n, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    for (size_t i = 0; i < n; ++i) {
      near_flag[i] = cs[i].nearBody ? 1 : 0;
      normal[3 * i] = cs[i].normal.x;
      normal[3 * i + 1] = cs[i].normal.y;
      normal[3 * i + 2] = cs[i].normal.z;
      offset[i] = cs[i].normal.w;
    }
  });
}

int drape_cuda_capture_system(drape_solver* s, double h, float* blocks, float* grad, uint8_t* active) {
  return guarded(s, [&] {
    need(s);
    s->requireBuilt();
    s->use();
    const size_t n = s->m.x.size();
    if (!n) return;
    // Run the substep prologue on scratch copies of the mutable state so the solver state is not changed.
    DBuf<float4> xs0, u0, ys0, xst0;
    DBuf<dcu::Contact> c0;
    xs0.alloc(n);
    c0.alloc(n);
    u0.alloc(n);
    ys0.alloc(n);
    xst0.alloc(n);
    CK(cudaMemcpyAsync(c0.p, s->contact.p, sizeof(dcu::Contact) * n, cudaMemcpyDeviceToDevice, s->stream));
    dcu::Control ctlSave{};
    CK(cudaMemcpyAsync(&ctlSave, s->ctl.p, sizeof(ctlSave), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    dcu::Dev d = s->dev;
    d.P.h = static_cast<float>(h);
    d.P.invH2 = static_cast<float>(1.0 / (h * h));
    d.P.hD = h;
    d.contact = c0.p;
    d.u = u0.p;
    d.yRel = ys0.p;
    d.xStart = xst0.p;
    const int pg = std::max<int>(1, static_cast<int>((n + 255) / 256));
    dcu::k_begin<<<pg, 256, 0, s->stream>>>(d);
    dcu::k_activate<<<pg, 256, 0, s->stream>>>(d);
    dcu::k_terms<<<s->termsGrid, dcu::kTermThreads, 0, s->stream>>>(d);
    dcu::k_assemble<<<s->assembleGrid, dcu::kAssembleThreads, 0, s->stream>>>(d);
    CK(cudaGetLastError());
    const size_t B = s->m.colIndex.size(), SP = s->dev.P.slotsPadded;
    std::vector<float> planes(9 * SP);
    std::vector<float4> g(n);
    std::vector<dcu::Contact> cs(n);
    CK(cudaMemcpyAsync(planes.data(), s->blocks.p, sizeof(float) * 9 * SP, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaMemcpyAsync(g.data(), s->grad.p, sizeof(float4) * n, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaMemcpyAsync(cs.data(), c0.p, sizeof(dcu::Contact) * n, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaMemcpyAsync(s->ctl.p, &ctlSave, sizeof(ctlSave), cudaMemcpyHostToDevice, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    for (size_t k = 0; k < B; ++k)
      for (int c = 0; c < 9; ++c) blocks[9 * k + c] = planes[c * SP + k];
    for (size_t i = 0; i < n; ++i) {
      grad[3 * i] = g[i].x;
      grad[3 * i + 1] = g[i].y;
      grad[3 * i + 2] = g[i].z;
      active[i] = cs[i].active ? 1 : 0;
    }
  });
}

int drape_cuda_pcg(uint32_t n, const uint32_t* row_start, const uint32_t* col_index, const float* blocks,
                   const uint8_t* pinned, const uint8_t* active, const float* normals, const float* grad,
                   int max_iterations, double tolerance, float* step, float* resid, int* iterations) {
  return guarded(nullptr, [&] {
    if (!row_start || !col_index || !blocks || !pinned || !grad || !step || !resid || !iterations)
      throw std::invalid_argument("null argument");
    int dev = 0;
    CK(cudaGetDevice(&dev));
    drape_solver s(dev);
    const uint32_t B = row_start[n];
    const uint32_t SP = (B + 31u) & ~31u;
    std::vector<uint32_t> cols(col_index, col_index + B);
    for (auto& c : cols) {
      if (c >= n) throw std::invalid_argument("column index out of range");
      if (pinned[c]) c |= dcu::kPinnedBit;
    }
    std::vector<float> planes(9 * static_cast<size_t>(SP), 0.0f);
    for (size_t k = 0; k < B; ++k)
      for (int c = 0; c < 9; ++c) planes[c * SP + k] = blocks[9 * k + c];
    std::vector<dcu::Particle> parts(n);
    std::vector<dcu::Contact> cs(n);
    std::vector<float4> g(n), pre(3 * static_cast<size_t>(n));
    for (uint32_t i = 0; i < n; ++i) {
      parts[i] = {1.0f, 0, 0, pinned[i] ? 1u : 0u};
      cs[i].active = active && active[i] ? 1u : 0u;
      cs[i].nearBody = cs[i].active;
      if (normals) cs[i].normal = make_float4(normals[3 * i], normals[3 * i + 1], normals[3 * i + 2], 0.0f);
      g[i] = make_float4(grad[3 * i], grad[3 * i + 1], grad[3 * i + 2], 0.0f);
      // Block-Jacobi inverse of the diagonal block, computed on the host here exactly as k_assemble does on the device
      // is not required: this entry point builds the preconditioner with the same device routine below.
    }
    cudaStream_t st = s.stream;
    DBuf<dcu::Particle> dpart;
    DBuf<uint32_t> drs, dci;
    DBuf<float> dbl;
    DBuf<float4> dg, dstep, dr, dz, dp0, dp1, dap, dapf, dres, dpre;
    DBuf<dcu::Contact> dcs;
    dpart.upload(parts, st);
    drs.upload(std::vector<uint32_t>(row_start, row_start + n + 1), st);
    dci.upload(cols, st);
    dbl.upload(planes, st);
    dg.upload(g, st);
    dcs.upload(cs, st);
    for (DBuf<float4>* b : {&dstep, &dr, &dz, &dp0, &dp1, &dap, &dapf, &dres}) b->alloc(n);
    dpre.alloc(3 * static_cast<size_t>(n));
    dcu::Dev d{};
    d.P.smemSlots = std::min(s.solveSmemCap, maxBlockSlots(row_start, n, s.solveGrid));
    d.P.n = n;
    d.P.nBlocks = B;
    d.P.slotsPadded = SP;
    d.P.maxCg = max_iterations;
    d.P.cgTolerance = tolerance;
    d.P.barrierLimitNs = s.barrierLimitNs;
    d.P.h = 1.0f;
    d.P.hD = 1.0;
    d.particle = dpart.p;
    d.rowStart = drs.p;
    d.colIndex = dci.p;
    d.blocks = dbl.p;
    d.grad = dg.p;
    d.contact = dcs.p;
    d.step = dstep.p;
    d.r = dr.p;
    d.z = dz.p;
    d.p0 = dp0.p;
    d.p1 = dp1.p;
    d.ap = dap.p;
    d.apFull = dapf.p;
    d.resid = dres.p;
    d.precond = dpre.p;
    d.partials = s.partials.p;
    d.ctl = s.ctl.p;
    // Preconditioner: diagonal block inverses with the device routine, then the persistent PCG alone (no line search:
    // the energy terms are absent, so k_solve stops after the contact-force phase with slope computed on zero terms).
    std::vector<uint32_t> diag(n, B);
    for (uint32_t i = 0; i < n; ++i)
      for (uint32_t k = row_start[i]; k < row_start[i + 1]; ++k)
        if (col_index[k] == i) diag[i] = k;
    for (uint32_t i = 0; i < n; ++i)
      if (diag[i] == B) throw std::invalid_argument("row without a diagonal block");
    DBuf<uint32_t> ddiag;
    ddiag.upload(diag, st);
    dcu::k_pcg_precondition<<<std::max<int>(1, static_cast<int>((n + 255) / 256)), 256, 0, st>>>(d, ddiag.p);
    CK(cudaGetLastError());
    void* args[] = {&d};
    CK(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(dcu::k_pcg_only), dim3(s.solveGrid),
                                   dim3(dcu::kSolveThreads), args,
                                   static_cast<size_t>(d.P.smemSlots) * dcu::kSmemSlotBytes, st));
    std::vector<float4> hs(n), hr(n);
    dcu::Control c{};
    CK(cudaMemcpyAsync(hs.data(), dstep.p, sizeof(float4) * n, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(hr.data(), dres.p, sizeof(float4) * n, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&c, s.ctl.p, sizeof(c), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (c.error) throw std::runtime_error("cuda: a grid barrier timed out");
    for (uint32_t i = 0; i < n; ++i) {
      step[3 * i] = hs[i].x;
      step[3 * i + 1] = hs[i].y;
      step[3 * i + 2] = hs[i].z;
      resid[3 * i] = hr[i].x;
      resid[3 * i + 1] = hr[i].y;
      resid[3 * i + 2] = hr[i].z;
    }
    *iterations = c.lastCg;
  });
}

int drape_cuda_spmv_device(uint32_t n, const uint32_t* d_row_start, const uint32_t* d_col_index, const float* d_blocks,
                           uint32_t slots_padded, const uint8_t* d_pinned, const void* d_x, void* d_y, void* stream) {
  return guarded(nullptr, [&] {
    if (!n) return;
    int dev = 0;
    CK(cudaGetDevice(&dev));
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const uint32_t blocksNeeded = (n + dcu::kSpmvBlockRows - 1) / dcu::kSpmvBlockRows;
    const uint32_t grid = std::min<uint32_t>(blocksNeeded, static_cast<uint32_t>(sms) * 64);
    dcu::k_spmv<<<grid, dcu::kSpmvThreads, 0, static_cast<cudaStream_t>(stream)>>>(
        n, d_row_start, d_col_index, d_blocks, slots_padded, d_pinned, static_cast<const float4*>(d_x),
        static_cast<float4*>(d_y));
    CK(cudaGetLastError());
  });
}

int drape_cuda_set_precond(drape_solver* s, drape_precond* p) {
  return guarded(s, [&] {
    need(s);
    s->use();
    s->setPrecond(p);
  });
}

int drape_cuda_precond_factor(drape_solver* s, float* l_blocks) {
  return guarded(s, [&] {
    need(s);
    s->requireBuilt();
    if (!l_blocks) throw std::invalid_argument("null argument");
    if (!s->netGraph) throw std::logic_error("the learned preconditioner is not in use");
    s->use();
    const net::Graph& g = s->net->graphOf(*s->netGraph);
    std::vector<float> planes(9 * static_cast<size_t>(g.SP));
    CK(cudaMemcpyAsync(planes.data(), g.L, sizeof(float) * planes.size(), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    for (uint32_t k = 0; k < g.B; ++k)
      for (int c = 0; c < 9; ++c) l_blocks[9 * static_cast<size_t>(k) + c] = planes[c * g.SP + k];
  });
}

int drape_cuda_set_precond_schedule(drape_solver* s, int refresh_every, int jacobi_first) {
  return guarded(s, [&] {
    need(s);
    if (refresh_every < 1) throw std::invalid_argument("refresh interval must be >= 1");
    if (jacobi_first < 0) throw std::invalid_argument("jacobi_first must be >= 0");
    s->precondRefresh = refresh_every;
    s->precondSwitch = jacobi_first;
  });
}

int drape_cuda_frame_times(drape_solver* s, uint64_t* begin_ns, uint64_t* end_ns, size_t capacity, size_t* count) {
  return guarded(s, [&] {
    need(s);
    if (!count || (capacity && (!begin_ns || !end_ns))) throw std::invalid_argument("null argument");
    const size_t k = std::min(capacity, s->frameTimes.size());
    for (size_t i = 0; i < k; ++i) {
      begin_ns[i] = s->frameTimes[i].first;
      end_ns[i] = s->frameTimes[i].second;
    }
    *count = k;
    s->frameTimes.clear();
  });
}

int drape_cuda_set_host_wait(drape_solver* s, uint32_t spin_microseconds) {
  return guarded(s, [&] {
    need(s);
    s->waitSpinUs = spin_microseconds;
  });
}

int drape_cuda_set_pcg_variant(drape_solver* s, int variant) {
  return guarded(s, [&] {
    need(s);
    if (variant < 0 || variant > 3)
      throw std::invalid_argument("PCG variant must be 0 (reference order), 1 (pipelined), 2 (Chronopoulos-Gear) or 3 "
                                  "(reference order, 1024-thread kernel)");
    s->pcgVariant = variant;
    s->dev.P.pcgVariant = variant;  // the frame graphs compare the device view and recapture
  });
}

int drape_cuda_solve_threads(const drape_solver* s, int* threads) {
  return guarded(s, [&] {
    need(s);
    if (!threads) throw std::invalid_argument("null argument");
    s->requireBuilt();
    *threads = s->usesResidentRows(s->dev) ? dcu::kRowThreads : dcu::kSolveThreads;
  });
}

int drape_cuda_set_barrier_limit(drape_solver* s, uint64_t nanoseconds) {
  return guarded(s, [&] {
    need(s);
    s->barrierLimitNs = nanoseconds ? nanoseconds : 2000000000ull;
  });
}

int drape_cuda_test_barrier_timeout(int device, int blocks, uint64_t nanoseconds, int* status) {
  return guarded(nullptr, [&] {
    if (!status || blocks < 1 || blocks > 1024) throw std::invalid_argument("bad argument");
    if (nanoseconds == 0 || nanoseconds > 1000000000ull) throw std::invalid_argument("limit must be in (0, 1 s]");
    CK(cudaSetDevice(device));
    DBuf<dcu::Control> c;
    DBuf<int> out;
    c.alloc(1);
    out.alloc(1);
    dcu::k_barrier_probe<<<blocks, 32>>>(c.p, nanoseconds, out.p);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    CK(cudaMemcpy(status, out.p, sizeof(int), cudaMemcpyDeviceToHost));
  });
}

int drape_cuda_reduction_floor(int device, int mode, int iterations, double* ns_per_iteration) {
  return guarded(nullptr, [&] {
    if (!ns_per_iteration || mode < 0 || mode > 7 || iterations < 1 || iterations > 1000000)
      throw std::invalid_argument("bad argument");
    const bool rows = mode >= 4;  // modes 4-7: modes 0-3 on k_solve_rows's 512-thread blocks
    mode &= 3;
    CK(cudaSetDevice(device));
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    DBuf<dcu::Control> c;
    DBuf<double> partials;
    DBuf<unsigned long long> out;
    c.alloc(1);
    partials.alloc(2 * static_cast<size_t>(sms) * dcu::kPartialStride);
    out.alloc(1);
    CK(cudaMemset(c.p, 0, sizeof(dcu::Control)));
    dcu::Dev d{};
    d.ctl = c.p;
    d.partials = partials.p;
    d.P.barrierLimitNs = 2000000000ull;
    unsigned long long* o = out.p;
    void* args[] = {&d, &mode, &iterations, &o};
    if (rows) {
      CK(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(dcu::k_reduction_floor<dcu::kRowThreads>), dim3(sms),
                                     dim3(dcu::kRowThreads), args, 0, nullptr));
    } else {
      CK(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(dcu::k_reduction_floor<dcu::kSolveThreads>), dim3(sms),
                                     dim3(dcu::kSolveThreads), args, 0, nullptr));
    }
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    unsigned long long ns = 0;
    dcu::Control h{};
    CK(cudaMemcpy(&ns, out.p, sizeof(ns), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&h, c.p, sizeof(h), cudaMemcpyDeviceToHost));
    if (h.error || ns == 0) throw std::runtime_error("cuda: a grid barrier timed out");
    *ns_per_iteration = static_cast<double>(ns) / iterations;
  });
}

int drape_cuda_inject_failure(drape_solver* s, int steps) {
  return guarded(s, [&] {
    need(s);
    s->failAfter = steps;
  });
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------------------------
// drape_cuda_pcg_noalloc: the PCG on caller-owned device buffers with all scratch in one file-scope device array.

namespace {

constexpr uint32_t kNoAllocMaxBlocks = 256;  // partials capacity (grid = one block per SM)

// Byte layout of the scratch array (every region 256-byte aligned).
struct NoAllocLayout {
  static constexpr size_t N = DRAPE_PCG_NOALLOC_MAX_PARTICLES, B = DRAPE_PCG_NOALLOC_MAX_SLOTS;
  static constexpr size_t vectors = 0;                                   // r, z, p0, p1, ap, apFull
  static constexpr size_t precond = vectors + 6 * sizeof(float4) * N;    // 3 float4 per particle
  static constexpr size_t particle = precond + 3 * sizeof(float4) * N;
  static constexpr size_t contact = particle + sizeof(dcu::Particle) * N;
  static constexpr size_t diag = contact + sizeof(dcu::Contact) * N;
  static constexpr size_t cols = diag + sizeof(uint32_t) * N;
  static constexpr size_t partials = cols + sizeof(uint32_t) * B;
  static constexpr size_t control = partials + 2 * kNoAllocMaxBlocks * dcu::kPartialStride * sizeof(double);
  static constexpr size_t total = control + 256;
};
static_assert(sizeof(dcu::Control) <= 256, "control block fits its region");
static_assert(NoAllocLayout::total == DRAPE_PCG_NOALLOC_SCRATCH_BYTES, "scratch size matches the header");

// The scratch. In host code this name is a host-side stand-in, not a device address: the address a kernel may use
// comes from cudaGetSymbolAddress (noAllocScratch() below).
__device__ __align__(256) unsigned char g_pcgScratch[NoAllocLayout::total];

struct NoAllocDevice {
  unsigned char* scratch = nullptr;
  int sms = 0;
  bool ready = false;
};
constexpr int kNoAllocMaxDevices = 64;
NoAllocDevice g_noAlloc[kNoAllocMaxDevices];
std::mutex g_noAllocMutex;

// The device address of the scratch array and the SM count, with `device` current. The SM count is looked up once per
// device. The address is looked up again on every call made outside a stream capture (cudaGetSymbolAddress allocates
// nothing), so a context that another framework re-created, or a cudaDeviceReset, leaves no stale address behind;
// during a capture the address from the last uncaptured call is used.
NoAllocDevice& noAllocScratch(int device, cudaStream_t stream) {
  if (device < 0 || device >= kNoAllocMaxDevices) throw std::runtime_error("cuda: device index out of range");
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  CK(cudaStreamIsCapturing(stream, &capture));
  std::lock_guard<std::mutex> lock(g_noAllocMutex);
  NoAllocDevice& d = g_noAlloc[device];
  if (!d.ready || capture == cudaStreamCaptureStatusNone) {
    if (!d.ready && capture != cudaStreamCaptureStatusNone)
      throw std::runtime_error("cuda: the first no-allocation PCG call on a device must come before any capture");
    void* p = nullptr;
    CK(cudaGetSymbolAddress(&p, g_pcgScratch));
    if (!d.ready) {
      CK(cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, device));
      if (d.sms < 1 || static_cast<uint32_t>(d.sms) > kNoAllocMaxBlocks)
        throw std::runtime_error("cuda: unsupported SM count for the no-allocation PCG");
    }
    d.scratch = static_cast<unsigned char*>(p);
    d.ready = true;
  }
  return d;
}

}  // namespace

namespace dcu {

// Error code in Control::error for a caller's block-CSR structure that the no-allocation PCG refuses: row_start not
// non-decreasing from 0 to `slots`, a column index >= n, or a row without its diagonal block.
constexpr int kNoAllocBadStructure = 3;

// Clears the control block and the iteration output before the structure check can raise an error in it.
__global__ void k_noalloc_clear(Control* ctl, int* iterations) {
  *ctl = Control{};
  *iterations = 0;
}

// Converts the caller's flags into the solver's layouts inside the scratch (particle pinned flags, contact state,
// columns with the pinned bit, diagonal slots) and checks the structure on the way. Every read and write stays in
// bounds whatever the caller passed: slot indices are clamped to [0, slots) and column indices are checked against n
// before they index `pinned`; a violation raises kNoAllocBadStructure and leaves in-range placeholders behind, which
// the solve never reads because it does not start.
__global__ void k_noalloc_prepare(uint32_t n, uint32_t slots, const uint32_t* __restrict__ rowStart,
                                  const uint32_t* __restrict__ colIndex, const uint8_t* __restrict__ pinned,
                                  const uint8_t* __restrict__ active, const float4* __restrict__ normals,
                                  Particle* particle, Contact* contact, uint32_t* cols, uint32_t* diag, Control* ctl) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  if (tid == 0 && (rowStart[0] != 0u || rowStart[n] != slots)) atomicExch(&ctl->error, kNoAllocBadStructure);
  for (uint32_t i = tid; i < n; i += stride) {
    particle[i] = Particle{1.0f, 0u, 0u, pinned[i] ? 1u : 0u};
    Contact c{};
    c.active = active && active[i] ? 1u : 0u;
    c.nearBody = c.active;
    if (normals) c.normal = make_float4(normals[i].x, normals[i].y, normals[i].z, 0.0f);
    contact[i] = c;
    const uint32_t rs = rowStart[i], re = rowStart[i + 1];
    bool bad = rs > re || re > slots;
    const uint32_t lo = min(rs, slots), hi = min(max(rs, re), slots);
    uint32_t d = slots;
    for (uint32_t s = lo; s < hi; ++s) {
      const uint32_t j = colIndex[s];
      if (j >= n) {
        bad = true;
        cols[s] = 0u;
        continue;
      }
      cols[s] = pinned[j] ? (j | kPinnedBit) : j;
      if (j == i) d = s;
    }
    if (d == slots) {
      bad = true;
      d = 0u;  // slots >= n >= 1 (checked on the host), so slot 0 exists
    }
    diag[i] = d;
    if (bad) atomicExch(&ctl->error, kNoAllocBadStructure);
  }
}

// k_pcg_precondition and k_pcg_only of the allocating entry point, skipped once the structure check has failed (every
// block reads the same flag, written by an earlier kernel on the stream, so the cooperative launch returns as a whole).
__global__ void k_noalloc_precondition(Dev D, const uint32_t* __restrict__ diag) {
  if (*reinterpret_cast<volatile int*>(&D.ctl->error) != 0) return;
  const uint32_t SP = D.P.slotsPadded;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < D.P.n; i += gridDim.x * blockDim.x) {
    M3 A;
#pragma unroll
    for (int k = 0; k < 9; ++k) A.m[k] = D.blocks[k * SP + diag[i]];
    M3 inv;
    if (D.particle[i].pinned != 0u) {
      zero(inv);
    } else {
      bool ok = false;
      inv = invertSpd(A, ok);
    }
    D.precond[3 * i + 0] = make_float4(inv.m[0], inv.m[1], inv.m[2], 0.0f);
    D.precond[3 * i + 1] = make_float4(inv.m[3], inv.m[4], inv.m[5], 0.0f);
    D.precond[3 * i + 2] = make_float4(inv.m[6], inv.m[7], inv.m[8], 0.0f);
  }
}

__global__ void __launch_bounds__(kSolveThreads, 1) k_noalloc_pcg(Dev D) {
  if (*reinterpret_cast<volatile int*>(&D.ctl->error) != 0) return;
  GridSync gs;
  gs.init(D.ctl, D.P.barrierLimitNs);
  const int it = pcgSolve<false, kRowLanes>(D, gs);
  if (it >= 0 && blockIdx.x == 0 && threadIdx.x == 0) D.ctl->lastCg = it;
}

// -2: the structure check failed; -1: a grid barrier gave up waiting; else the PCG iteration count.
__global__ void k_noalloc_finish(const Control* ctl, int* iterations) {
  const int e = ctl->error;
  *iterations = e == kNoAllocBadStructure ? -2 : (e ? -1 : ctl->lastCg);
}

}  // namespace dcu

extern "C" int drape_cuda_pcg_noalloc(uint32_t n, uint32_t slots, const uint32_t* d_row_start,
                                      const uint32_t* d_col_index, const float* d_blocks, uint32_t slots_padded,
                                      const uint8_t* d_pinned, const uint8_t* d_active, const void* d_normals,
                                      const void* d_grad, int max_iterations, double tolerance, void* d_step,
                                      void* d_resid, int32_t* d_iterations, void* stream) {
  return guarded(nullptr, [&] {
    if (n == 0 || n > DRAPE_PCG_NOALLOC_MAX_PARTICLES)
      throw std::invalid_argument("pcg_noalloc: n must be in 1.." + std::to_string(DRAPE_PCG_NOALLOC_MAX_PARTICLES) +
                                  " (got " + std::to_string(n) + ")");
    if (!d_row_start || !d_col_index || !d_blocks || !d_pinned || !d_grad || !d_step || !d_resid || !d_iterations)
      throw std::invalid_argument("pcg_noalloc: null device pointer");
    if (max_iterations < 0) throw std::invalid_argument("pcg_noalloc: negative iteration cap");
    auto st = static_cast<cudaStream_t>(stream);
    if (slots > DRAPE_PCG_NOALLOC_MAX_SLOTS)
      throw std::invalid_argument("pcg_noalloc: " + std::to_string(slots) + " block slots exceed the limit of " +
                                  std::to_string(DRAPE_PCG_NOALLOC_MAX_SLOTS));
    if (slots < n) throw std::invalid_argument("pcg_noalloc: fewer block slots than rows (every row has a diagonal)");
    if (slots_padded < slots) throw std::invalid_argument("pcg_noalloc: slots_padded < row_start[n]");
    int device = 0;
    CK(cudaGetDevice(&device));
    NoAllocDevice& nd = noAllocScratch(device, st);
    unsigned char* base = nd.scratch;
    using L = NoAllocLayout;
    auto* vec = reinterpret_cast<float4*>(base + L::vectors);
    const size_t N = L::N;
    dcu::Dev d{};
    d.P.n = n;
    d.P.nBlocks = slots;
    d.P.slotsPadded = slots_padded;
    d.P.maxCg = max_iterations;
    d.P.cgTolerance = tolerance;
    d.P.barrierLimitNs = 2000000000ull;
    d.P.h = 1.0f;
    d.P.hD = 1.0;
    d.r = vec;
    d.z = vec + N;
    d.p0 = vec + 2 * N;
    d.p1 = vec + 3 * N;
    d.ap = vec + 4 * N;
    d.apFull = vec + 5 * N;
    d.precond = reinterpret_cast<float4*>(base + L::precond);
    d.particle = reinterpret_cast<const dcu::Particle*>(base + L::particle);
    d.contact = reinterpret_cast<dcu::Contact*>(base + L::contact);
    d.rowStart = d_row_start;
    d.colIndex = reinterpret_cast<const uint32_t*>(base + L::cols);
    d.blocks = const_cast<float*>(d_blocks);
    d.grad = const_cast<float4*>(static_cast<const float4*>(d_grad));
    d.step = static_cast<float4*>(d_step);
    d.resid = static_cast<float4*>(d_resid);
    d.partials = reinterpret_cast<double*>(base + L::partials);
    d.ctl = reinterpret_cast<dcu::Control*>(base + L::control);
    auto* diag = reinterpret_cast<uint32_t*>(base + L::diag);
    const int pg = std::max(1, static_cast<int>((n + 255) / 256));
    dcu::k_noalloc_clear<<<1, 1, 0, st>>>(d.ctl, d_iterations);
    CK(cudaGetLastError());
    dcu::k_noalloc_prepare<<<pg, 256, 0, st>>>(
        n, slots, d_row_start, d_col_index, d_pinned, d_active, static_cast<const float4*>(d_normals),
        reinterpret_cast<dcu::Particle*>(base + L::particle), d.contact, reinterpret_cast<uint32_t*>(base + L::cols),
        diag, d.ctl);
    CK(cudaGetLastError());
    dcu::k_noalloc_precondition<<<pg, 256, 0, st>>>(d, diag);
    CK(cudaGetLastError());
    void* args[] = {&d};
    CK(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(dcu::k_noalloc_pcg), dim3(nd.sms),
                                   dim3(dcu::kSolveThreads), args, 0, st));
    dcu::k_noalloc_finish<<<1, 1, 0, st>>>(d.ctl, d_iterations);
    CK(cudaGetLastError());
  });
}
