// The circle commit workload as one device-resident plan: circle LDE of all
// columns, row-leaf Merkle tree fused with the gamma combination and the layer-0
// FRI commitment, then the fold chain with one fused fold+commit launch per layer.
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
  ZS_CUDA(cudaStreamSynchronize(setup));
}

CommitPlan::~CommitPlan() {
  cudaDeviceSynchronize();
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
  cudaStreamDestroy(setup);
}

void CommitPlan::set_challenges(const uint32_t* h_gammas, const uint32_t* h_alphas) {
  std::vector<qm31> g(C);
  for (uint32_t c = 0; c < C; ++c) g[c] = qmake(h_gammas[4 * c], h_gammas[4 * c + 1], h_gammas[4 * c + 2], h_gammas[4 * c + 3]);
  for (unsigned i = 0; i < F; ++i)
    alphas[i] = qmake(h_alphas[4 * i], h_alphas[4 * i + 1], h_alphas[4 * i + 2], h_alphas[4 * i + 3]);
  ZS_CUDA(cudaMemcpy(gammas, g.data(), C * sizeof(qm31), cudaMemcpyHostToDevice));
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

void CommitPlan::run(const uint32_t* d_trace, cudaStream_t st) {
  run_phase(PHASE_LDE, d_trace, st);
  run_phase(PHASE_ROW_TREE, d_trace, st);
  run_phase(PHASE_FOLDS, d_trace, st);
}

uint32_t CommitPlan::launches() const {
  // circle_lde: 3; row tree: leaf kernel + tree_up launches (+ those of the g tree);
  // each fold: 1 + tree_up launches of the next layer's tree.
  auto up = [](unsigned log_n, unsigned from) {
    uint32_t k = 0;
    unsigned lvl = from;
    while (lvl < log_n) {
      const uint64_t count = (uint64_t)1 << (log_n - lvl);
      const uint64_t per = count >= 512 ? 512 : count;
      unsigned g = 0;
      while (((uint64_t)1 << g) < per) ++g;
      lvl += g;
      ++k;
    }
    return k;
  };
  auto run_log = [](uint64_t count) {
    const uint64_t threads = count >= 256 ? 256 : count;
    unsigned g = 0;
    while (((uint64_t)1 << g) < threads) ++g;
    return g;
  };
  const unsigned LB = L + B;
  uint32_t k = 3 + 1 + up(LB, run_log((uint64_t)1 << LB));
  if (F > 0) k += up(LB, run_log((uint64_t)1 << LB));
  for (unsigned i = 0; i < F; ++i) {
    k += 1;
    if (i + 1 < F) k += up(LB - i - 1, run_log((uint64_t)1 << (LB - i - 1)));
  }
  return k;
}

}  // namespace zs
