// The circle commit workload as one device-resident plan: circle LDE of all
// columns, row-leaf Merkle tree fused with the gamma combination and the layer-0
// FRI commitment, then the fold chain with one fused fold+commit launch per layer.
#include <algorithm>
#include <cstdlib>
#include <functional>
#include <memory>
#include <vector>

#include "circle.cuh"
#include "commit.cuh"
#include "fri.cuh"

namespace zs {

CommitPlan::CommitPlan(uint32_t C_, unsigned L_, unsigned B_, unsigned F_) : C(C_), L(L_), B(B_), F(F_) {
  if (C == 0 || C > 256) throw Error(ZS_EMALFORMED, "n_columns must be in [1, 256]");
  if (L < 1 || L + B > 28) throw Error(ZS_EMALFORMED, "log_rows + log_blowup must be in [1, 28]");
  if (F > L + B) throw Error(ZS_EMALFORMED, "more folds than domain bits");
  ZS_CUDA(cudaStreamCreateWithFlags(&setup, cudaStreamNonBlocking));
  ZS_CUDA(cudaStreamCreateWithFlags(&copy, cudaStreamNonBlocking));
  for (auto& s : sides) ZS_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  // Group sizes grow by about 4/3 from 2 columns at the end, so each group's LDE is
  // done before the next group's copy (the LDE of a column takes about 0.6 of its
  // copy over PCIe) and the step waits for a small group's LDE after the last copy.
  for (uint32_t g = 2, used = 0; used < C; g = std::max(g + 1, (g * 4 + 2) / 3)) {
    upload_groups.push_back(std::min(g, C - used));
    used += upload_groups.back();
  }
  std::sort(upload_groups.begin(), upload_groups.end(), std::greater<uint32_t>());
  up_events.resize(upload_groups.size() + 1);
  for (auto& e : up_events) ZS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  events.resize(F + 2 + kSides);
  for (auto& e : events) ZS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  const size_t n = (size_t)1 << L, N = (size_t)1 << (L + B);
  small = std::make_unique<CircleDomain>(L, setup);
  big = std::make_unique<CircleDomain>(L + B, setup);
  tabs = std::make_unique<FoldTables>(L + B, setup);
  auto alloc = [&](void** p, size_t bytes) { ZS_CUDA(cudaMallocAsync(p, bytes, setup)); };
  alloc((void**)&trace, C * n * sizeof(uint32_t));
  alloc((void**)&lde, C * N * sizeof(uint32_t));
  alloc((void**)&scratch, lde_scratch_words(L, B, C) * sizeof(uint32_t));
  alloc((void**)&gammas, C * sizeof(qm31));
  layers.resize(F + 1);
  for (unsigned i = 0; i <= F; ++i) alloc((void**)&layers[i], (N >> i) * sizeof(qm31));
  row_tree.log_n = L + B;
  alloc((void**)&row_tree.words, DeviceTree::words_for(L + B) * sizeof(uint32_t));
  layer_trees.resize(F);
  for (unsigned i = 0; i < F; ++i) {
    layer_trees[i].log_n = L + B - i;
    alloc((void**)&layer_trees[i].words, DeviceTree::words_for(L + B - i) * sizeof(uint32_t));
  }
  alphas.assign(F, qzero());
  const char* env = std::getenv("ZS_NO_GRAPH");
  use_graph = !(env && env[0] == '1');
  ZS_CUDA(cudaStreamSynchronize(setup));
}

CommitPlan::~CommitPlan() {
  cudaDeviceSynchronize();
  drop_graph();
  cudaFree(trace);
  cudaFree(lde);
  cudaFree(scratch);
  cudaFree(gammas);
  for (auto* p : layers) cudaFree(p);
  cudaFree(row_tree.words);
  for (auto& t : layer_trees) cudaFree(t.words);
  small.reset();
  big.reset();
  tabs.reset();
  for (auto& e : events) cudaEventDestroy(e);
  for (auto& e : up_events) cudaEventDestroy(e);
  cudaStreamDestroy(copy);
  for (auto& s : sides) cudaStreamDestroy(s);
  cudaStreamDestroy(setup);
}

void CommitPlan::set_challenges(const uint32_t* h_gammas, const uint32_t* h_alphas) {
  std::vector<qm31> g(C);
  for (uint32_t c = 0; c < C; ++c) g[c] = qmake(h_gammas[4 * c], h_gammas[4 * c + 1], h_gammas[4 * c + 2], h_gammas[4 * c + 3]);
  for (unsigned i = 0; i < F; ++i)
    alphas[i] = qmake(h_alphas[4 * i], h_alphas[4 * i + 1], h_alphas[4 * i + 2], h_alphas[4 * i + 3]);
  ZS_CUDA(cudaMemcpy(gammas, g.data(), C * sizeof(qm31), cudaMemcpyHostToDevice));
  drop_graph();  // fold challenges are baked into the captured launches
}

void CommitPlan::run_phase(int phase, const uint32_t* d_trace, cudaStream_t st) {
  const size_t n = (size_t)1 << L, N = (size_t)1 << (L + B);
  if (!d_trace) d_trace = trace;
  switch (phase) {
    case PHASE_LDE:
      circle_lde(d_trace, n, lde, N, C, L, B, *small, *big, scratch, st);
      break;
    case PHASE_ROW_TREE:
      build_row_tree(lde, N, C, row_tree, gammas, layers[0], F > 0 ? &layer_trees[0] : nullptr, st);
      break;
    case PHASE_FOLDS:
      for (unsigned i = 0; i < F; ++i) {
        const uint32_t half = (uint32_t)(N >> (i + 1));
        fri_fold(layers[i], layers[i + 1], half, alphas[i], i, *tabs, i + 1 < F ? &layer_trees[i + 1] : nullptr, st);
      }
      break;
    default:
      throw Error(ZS_EMALFORMED, "unknown phase");
  }
}

// The step as a DAG: the LDE, the row leaves and the fold chain run on `st`; each
// tree above its leaves (the row tree, the g tree, every committed fold layer's
// tree) is finished on a side stream as soon as its leaves exist, so the narrow
// tops of the trees overlap with each other and with the folds.
void CommitPlan::run_direct(const uint32_t* d_trace, cudaStream_t st) {
  const size_t n = (size_t)1 << L, N = (size_t)1 << (L + B);
  if (!d_trace) d_trace = trace;
  circle_lde(d_trace, n, lde, N, C, L, B, *small, *big, scratch, st);
  after_lde(st);
}

// Column group g is copied on `copy` and its LDE waits for that copy only; the groups'
// LDEs run in order on `st` and share the scratch buffer (sized for all C columns).
void CommitPlan::run_host_direct(const uint32_t* h_trace, cudaStream_t st) {
  const size_t n = (size_t)1 << L, N = (size_t)1 << (L + B);
  const size_t G = upload_groups.size();
  ZS_CUDA(cudaEventRecord(up_events[G], st));  // the previous step is done with `trace`
  ZS_CUDA(cudaStreamWaitEvent(copy, up_events[G], 0));
  for (size_t g = 0, c0 = 0; g < G; c0 += upload_groups[g++]) {
    ZS_CUDA(cudaMemcpyAsync(trace + c0 * n, h_trace + c0 * n, (size_t)upload_groups[g] * n * sizeof(uint32_t),
                            cudaMemcpyHostToDevice, copy));
    ZS_CUDA(cudaEventRecord(up_events[g], copy));
  }
  for (size_t g = 0, c0 = 0; g < G; c0 += upload_groups[g++]) {
    ZS_CUDA(cudaStreamWaitEvent(st, up_events[g], 0));
    circle_lde(trace + c0 * n, n, lde + c0 * N, N, upload_groups[g], L, B, *small, *big, scratch, st);
  }
  after_lde(st);
}

void CommitPlan::run_host(const uint32_t* h_trace, cudaStream_t st) {
  if (!use_graph) return run_host_direct(h_trace, st);
  if (!host_exec || host_trace != h_trace) {
    if (host_exec) cudaGraphExecDestroy(host_exec);
    host_exec = nullptr;
    cudaGraph_t g = nullptr;
    ZS_CUDA(cudaStreamBeginCapture(setup, cudaStreamCaptureModeThreadLocal));
    try {
      run_host_direct(h_trace, setup);
    } catch (...) {
      cudaStreamEndCapture(setup, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    ZS_CUDA(cudaStreamEndCapture(setup, &g));
    const cudaError_t e = cudaGraphInstantiate(&host_exec, g, 0);
    cudaGraphDestroy(g);
    ZS_CUDA(e);
    host_trace = h_trace;
  }
  ZS_CUDA(cudaGraphLaunch(host_exec, st));
}

// Everything after the LDE: row leaves with the gamma combination, the trees, the folds.
void CommitPlan::after_lde(cudaStream_t st) {
  const size_t N = (size_t)1 << (L + B);
  build_row_leaves(lde, N, C, row_tree, gammas, layers[0], F > 0 ? &layer_trees[0] : nullptr, st);
  unsigned side = 0;
  bool used[kSides] = {};
  auto branch = [&](DeviceTree& t) {
    cudaEvent_t e = events[ev_used++];
    ZS_CUDA(cudaEventRecord(e, st));
    used[side % kSides] = true;
    cudaStream_t s = sides[side++ % kSides];
    ZS_CUDA(cudaStreamWaitEvent(s, e, 0));
    tree_finish(t, 0, s);
  };
  ev_used = 0;
  branch(row_tree);
  if (F > 0) branch(layer_trees[0]);
  for (unsigned i = 0; i < F; ++i) {
    const uint32_t half = (uint32_t)(N >> (i + 1));
    const bool commit = i + 1 < F;
    fri_fold(layers[i], layers[i + 1], half, alphas[i], i, *tabs, commit ? &layer_trees[i + 1] : nullptr, st,
             /*finish_tree=*/false);
    if (commit) branch(layer_trees[i + 1]);
  }
  for (unsigned k = 0; k < kSides; ++k) {
    if (!used[k]) continue;  // only streams forked from `st` may join it (graph capture)
    cudaEvent_t e = events[ev_used++];
    ZS_CUDA(cudaEventRecord(e, sides[k]));
    ZS_CUDA(cudaStreamWaitEvent(st, e, 0));
  }
}

void CommitPlan::drop_graph() {
  if (graph_exec) cudaGraphExecDestroy(graph_exec);
  graph_exec = nullptr;
  graph_trace = nullptr;
  if (host_exec) cudaGraphExecDestroy(host_exec);
  host_exec = nullptr;
  host_trace = nullptr;
}

// The whole step is one CUDA graph (about a hundred launches, most of them small
// tree and fold kernels), captured on the plan's own stream and replayed on the
// caller's; it is recaptured when the trace pointer or the challenges change.
void CommitPlan::run(const uint32_t* d_trace, cudaStream_t st) {
  if (!d_trace) d_trace = trace;
  if (!use_graph) return run_direct(d_trace, st);
  if (!graph_exec || graph_trace != d_trace) {
    drop_graph();
    cudaGraph_t g = nullptr;
    ZS_CUDA(cudaStreamBeginCapture(setup, cudaStreamCaptureModeThreadLocal));
    try {
      run_direct(d_trace, setup);
    } catch (...) {
      cudaStreamEndCapture(setup, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    ZS_CUDA(cudaStreamEndCapture(setup, &g));
    const cudaError_t e = cudaGraphInstantiate(&graph_exec, g, 0);
    cudaGraphDestroy(g);
    ZS_CUDA(e);
    graph_trace = d_trace;
  }
  ZS_CUDA(cudaGraphLaunch(graph_exec, st));
}

uint32_t CommitPlan::launches() const {
  // circle_lde: 3; row leaves: 1 + the row tree's and the g tree's tree_finish;
  // each fold: 1 + the folded layer's tree_finish when it is committed.
  const unsigned LB = L + B;
  uint32_t k = 3 + 1 + tree_finish_launches(LB, 0);
  if (F > 0) k += tree_finish_launches(LB, 0);
  for (unsigned i = 0; i < F; ++i) k += 1 + (i + 1 < F ? tree_finish_launches(LB - i - 1, 0) : 0);
  return k;
}

}  // namespace zs
