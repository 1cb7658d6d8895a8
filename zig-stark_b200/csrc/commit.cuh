// Device-resident plan of the circle commit workload (see commit.cu).
#pragma once
#include <memory>
#include <vector>

#include "circle.cuh"
#include "fri.cuh"
#include "merkle.cuh"

namespace zs {

enum CommitPhase : int { PHASE_LDE = 0, PHASE_ROW_TREE = 1, PHASE_FOLDS = 2 };

struct CommitPlan {
  uint32_t C;
  unsigned L, B, F;
  cudaStream_t setup = nullptr;
  std::unique_ptr<CircleDomain> small, big;
  std::unique_ptr<FoldTables> tabs;
  uint32_t* trace = nullptr;    // C x 2^L, column-major
  uint32_t* lde = nullptr;      // C x 2^(L+B), column-major, natural order
  uint32_t* scratch = nullptr;  // circle_lde scratch
  qm31* gammas = nullptr;       // C
  std::vector<qm31> alphas;     // F, host
  std::vector<qm31*> layers;    // F + 1 fold layers; layers[0] = g
  DeviceTree row_tree;
  std::vector<DeviceTree> layer_trees;  // trees of layers 0 .. F-1

  CommitPlan(uint32_t C, unsigned L, unsigned B, unsigned F);
  ~CommitPlan();
  CommitPlan(const CommitPlan&) = delete;
  CommitPlan& operator=(const CommitPlan&) = delete;
  void set_challenges(const uint32_t* h_gammas, const uint32_t* h_alphas);
  // Replays the captured graph of the whole step (set ZS_NO_GRAPH=1 for direct launches).
  void run(const uint32_t* d_trace, cudaStream_t st);
  void run_direct(const uint32_t* d_trace, cudaStream_t st);
  // One of the three phases of run(): the circle LDE (3 launches); the row-leaf
  // tree fused with the gamma combination and the layer-0 tree; the fold chain.
  void run_phase(int phase, const uint32_t* d_trace, cudaStream_t st);
  uint32_t launches() const;
  // The step from a trace in pinned host memory: column groups are copied on a copy
  // stream while the LDE of the groups already on the device runs, then the rest of
  // the step; replayed as one captured graph per host pointer.
  void run_host(const uint32_t* h_trace, cudaStream_t st);
  void run_host_direct(const uint32_t* h_trace, cudaStream_t st);
  // Column counts of the upload groups, largest first: after the last copy only the
  // last (smallest) group's LDE precedes the rest of the step.
  std::vector<uint32_t> upload_groups;

 private:
  static constexpr unsigned kSides = 3;
  cudaStream_t sides[kSides] = {};
  std::vector<cudaEvent_t> events;
  unsigned ev_used = 0;
  bool use_graph = true;
  cudaGraphExec_t graph_exec = nullptr;
  const uint32_t* graph_trace = nullptr;
  cudaStream_t copy = nullptr;
  std::vector<cudaEvent_t> up_events;  // one per upload group, plus one
  cudaGraphExec_t host_exec = nullptr;
  const uint32_t* host_trace = nullptr;
  void drop_graph();
  void after_lde(cudaStream_t st);
};

}  // namespace zs
