// Learned preconditioner: a message-passing network over the block-CSR graph of a Newton system that emits the
// block lower-triangular factor L of M^-1 = L L^T (L = S G with S = blockdiag(chol(inv(A_ii))); G = I is block-Jacobi
// exactly). Forward and backward run as tcgen05 tile kernels (BF16 operands in shared memory, FP32 accumulators in
// TMEM); the optimiser is Adam on FP32 master weights. No counterpart in the reference, whose PCG is block-Jacobi
// (cpu_solver.cpp:169-213).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

namespace net {

constexpr int kHidden = 64;
constexpr int kLayers = 4;
constexpr int kNodeFeatures = 16;
constexpr int kEdgeFeatures = 16;
constexpr int kOutputs = 16;
constexpr int kTileSlots = 128;  // slots per row tile (rows are packed whole)
constexpr float kAggScale = 0.125f;
constexpr float kDiagClamp = 8.0f;

// Flat parameter layout ([out][in] row-major weights, then the bias), in this order: W_ne b_ne W_ee b_ee, per layer
// W_m b_m W_u b_u, then W_o b_o.
struct Layout {
  static constexpr size_t kNe = 0, kNeB = kNe + kHidden * kNodeFeatures;
  static constexpr size_t kEe = kNeB + kHidden, kEeB = kEe + kHidden * kEdgeFeatures;
  static constexpr size_t kLayer0 = kEeB + kHidden;
  static constexpr size_t kLayerSize = 2 * (kHidden * 2 * kHidden + kHidden);
  __host__ __device__ static constexpr size_t m(int l) { return kLayer0 + l * kLayerSize; }
  __host__ __device__ static constexpr size_t mB(int l) { return m(l) + kHidden * 2 * kHidden; }
  __host__ __device__ static constexpr size_t u(int l) { return mB(l) + kHidden; }
  __host__ __device__ static constexpr size_t uB(int l) { return u(l) + kHidden * 2 * kHidden; }
  static constexpr size_t kO = kLayer0 + kLayers * kLayerSize, kOB = kO + kOutputs * 3 * kHidden;
  static constexpr size_t kCount = kOB + kOutputs;
};

// Device view of one graph (a Newton system) and its network workspace.
struct Graph {
  uint32_t n = 0, B = 0, SP = 0, nTiles = 0;
  const uint32_t* rowStart = nullptr;
  const uint32_t* colIndex = nullptr;  // may carry the solver's pinned bit (bit 31)
  const uint32_t* tslot = nullptr;     // slot of (j, i) for slot (i, j)
  const uint32_t* tileRow = nullptr;   // nTiles + 1 row boundaries of the row tiles
  const float* blocks = nullptr;       // 9 planes of SP floats (component 3 * r + c of every slot)
  const uint8_t* pinnedBase = nullptr;  // pinned flag of row i at pinnedBase[i * pinnedStride] (nonzero: pinned)
  uint32_t pinnedStride = 1;
  const uint8_t* activeBase = nullptr;  // contact-active flag of row i at activeBase[i * activeStride]
  uint32_t activeStride = 1;
  // Workspace.
  float* C = nullptr;                // n x 9: chol(inv(A_ii)), row-major
  float* Ahat = nullptr;             // B x 9: C_i^T A_ij C_j
  __nv_bfloat16* f = nullptr;        // n x 16
  __nv_bfloat16* e = nullptr;        // B x 16
  __nv_bfloat16* eps = nullptr;      // B x 64
  __nv_bfloat16* h[kLayers + 1] = {};  // n x 64 per layer input (inference ping-pongs h[0] and h[1])
  __nv_bfloat16* agg[kLayers] = {};    // n x 64, a_i / 8 as staged (training only)
  float* G = nullptr;                // B x 9 (training only; lower live slots)
  float* o = nullptr;                // B x 16 (training only)
  float* L = nullptr;                // 9 planes of SP floats: the factor L = S G on lower live slots
  // Inference workspace (forwardOn without training; eps, Ahat and the per-layer h are not kept).
  __nv_bfloat16* E = nullptr;        // kLayers planes of B x 64: W_me^l eps_s + b_m^l
  float* F = nullptr;                // B x 16: W_oe eps_s + b_o
  __nv_bfloat16* P = nullptr;        // n x 64: W_mh^l h_j of the current layer
  float* Q = nullptr;                // n x 32: W_oi h_i (0..15), W_oj h_j (16..31)
  __nv_bfloat16* a = nullptr;        // n x 64: a_i of the current layer
  uint32_t* code = nullptr;          // B: column of the slot, bit 31 when either row is pinned (written by k_features)
  uint32_t* slotRow = nullptr;       // B: row of the slot (fixed with the CSR)
  const void* tmaps = nullptr;       // host memory: the TMA store maps of E and F (CUtensorMap[2])
  // A solver's bound graph only: per slot three float4 rows of a factor block for the solver's own products: L_ij at
  // the lower slots (j <= i) and, at each upper slot (i, j), L_ji (the block of its transposed slot).
  float4* LF = nullptr;
};

// Host-owned device buffers of a graph built from host arrays (a training sample) or bound to a solver's arrays.
struct GraphStore;
struct GraphStoreDeleter {
  void operator()(GraphStore* s) const;
};
using GraphHandle = std::unique_ptr<GraphStore, GraphStoreDeleter>;

class Network {
 public:
  explicit Network(int device);
  ~Network();
  Network(const Network&) = delete;
  Network& operator=(const Network&) = delete;

  void setParams(const float* p, size_t count);
  void getParams(float* p, size_t count);
  cudaStream_t stream() const { return stream_; }

  // Training samples (systems from host arrays, blocks row-major 9 per slot, residuals 3n each).
  int addSample(uint32_t n, const uint32_t* rowStart, const uint32_t* colIndex, const float* blocks,
                const uint8_t* pinned, const uint8_t* active, const float* residuals, uint32_t residualCount);
  void clearSamples();
  int sampleCount() const;

  void forward(int sample, float* Gout, float* Lout);                    // host copies (B x 9 each, row-major)
  double lossGrad(int sample, int residual, float* grad, bool accumulate);  // grad (host, count) may be null
  void apply(int sample, const float* r, float* z);                        // z = L L^T r (host, 3n each)
  void train(int steps, float lr, int batch, uint64_t seed, float* losses);
  // PCG on a sample's scaled system with residual `rhs` as the right-hand side; returns the iterations.
  int pcg(int sample, int rhs, bool useLearned, int maxIterations, double tolerance, double* relres);
  // 0: residual defect |Ahat G G^T rhat - rhat|^2 / |rhat|^2; 1: stochastic Kaporin objective on the probe vectors.
  void setObjective(int objective) { objective_ = objective; }

  // Forward on a solver's system: writes g.L (and the workspace) on `st`. Params must be set. A tensor-core wait that
  // gives up raises *error (the network's own flag when null). training: the fused tile kernels, keeping every
  // activation the backward pass reads; otherwise the inference path (needs the inference workspace).
  void forwardOn(Graph& g, cudaStream_t st, bool training, int* error = nullptr);
  // The inference path on a training sample (its inference workspace is allocated on first use); L as in forward.
  void forwardInference(int sample, float* Lout);
  // Builds a graph workspace for a solver's CSR (device arrays owned by the solver); returns the store to keep.
  GraphHandle bind(uint32_t n, uint32_t B, uint32_t SP, const uint32_t* hostRowStart,
                                   const uint32_t* hostColIndex, const uint32_t* dRowStart, const uint32_t* dColIndex,
                                   const float* dBlocks, const uint8_t* pinnedBase, uint32_t pinnedStride,
                                   const uint8_t* activeBase, uint32_t activeStride, cudaStream_t st,
                                   bool factorRows = false);  // factorRows: also keep Graph::LF (a solver's graph)
  Graph& graphOf(GraphStore& s);
  const __nv_bfloat16* weights() const { return wBf16_; }
  const float* master() const { return master_; }

 private:
  void lossForward(GraphStore& s, int residual);
  void backward(GraphStore& s);
  void reduceInto(const float* partials, int grid, size_t count, size_t offset, float scale);
  double lossValue(const GraphStore& s, const double* scalars) const;

  int device_;
  int numSMs_ = 0;
  cudaStream_t stream_ = nullptr;
  float* master_ = nullptr;        // FP32 master parameters
  __nv_bfloat16* wBf16_ = nullptr;  // BF16 copy the kernels read
  float* grad_ = nullptr;          // FP32 gradient accumulator
  float* adamM_ = nullptr;
  float* adamV_ = nullptr;
  float* partials_ = nullptr;      // per-CTA weight-gradient partials
  size_t partialsCount_ = 0;
  int* error_ = nullptr;           // device error flag (bounded waits)
  double* scalars_ = nullptr;      // device FP64 scratch (norms, loss)
  int adamStep_ = 0;
  int objective_ = 1;
  std::vector<std::unique_ptr<GraphStore>> samples_;
};

// Host helpers shared with the solver.
std::vector<uint32_t> rowTiles(const std::vector<uint32_t>& rowStart);
std::vector<uint32_t> transposedSlots(const std::vector<uint32_t>& rowStart, const std::vector<uint32_t>& colIndex);

}  // namespace net

// The C ABI's handle (include/drape_precond.h).
struct drape_precond {
  std::unique_ptr<net::Network> net;
  std::string error;
};
