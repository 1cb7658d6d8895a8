// Merkle trees (src/core/merkle/merkle.zig) built on the device.
#pragma once
#include <vector>

#include "common.cuh"

namespace zs {

// All levels of a tree over 2^log_n leaves in one buffer: level k (2^(log_n-k)
// digests) starts at digest 2N - (2N >> k), so the leaves come first and the root
// is the last digest. Digests are 8 little-endian u32 words (the Blake3 bytes).
struct DeviceTree {
  unsigned log_n = 0;
  uint32_t* words = nullptr;  // (2N - 1) * 8 words
  bool owned = false;
  static size_t words_for(unsigned log_n) { return (((size_t)2 << log_n) - 1) * 8; }
  size_t level_offset(unsigned k) const {
    const size_t N2 = (size_t)2 << log_n;
    return N2 - (N2 >> k);
  }
  const uint32_t* level(unsigned k) const { return words + 8 * level_offset(k); }
  uint32_t* level(unsigned k) { return words + 8 * level_offset(k); }
  const uint32_t* root() const { return level(log_n); }
};

// Leaves hashQM31(values[i]) for 2^log_n QM31 values plus the whole tree.
void build_qm31_tree(const qm31* d_values, DeviceTree& tree, cudaStream_t st);

// Device tree pointers of a set of trees built by the same launches (blockIdx.y picks
// the tree): small trees are latency-bound, so one launch per level range serves all.
constexpr uint32_t kTreeBatch = 64;
struct TreeSet {
  uint32_t* words[kTreeBatch];
};
// build_qm31_tree for `count` trees of one size: tree k over the values at
// d_values + k * v_stride.
void build_qm31_trees(const qm31* d_values, size_t v_stride, DeviceTree* const* trees, uint32_t count,
                      cudaStream_t st);
// Leaves only (level 0) of build_qm31_tree.
void build_qm31_leaves(const qm31* d_values, DeviceTree& tree, cudaStream_t st);
// Completes levels above `from_level` (levels <= from_level must be written), three
// levels per launch.
void tree_finish(DeviceTree& tree, unsigned from_level, cudaStream_t st);
// Number of launches tree_finish makes.
uint32_t tree_finish_launches(unsigned log_n, unsigned from_level);

// Opening path of leaf `index` (siblings bottom-up, merkle.zig:57-68), read back to
// the host from a device tree. `out` receives log_n digests of 32 bytes.
void tree_open_host(const DeviceTree& tree, uint64_t index, uint8_t* out, cudaStream_t st);

// Gathers `count` opening paths at once: out[q] = path of indices[q] (log_n * 32 bytes each).
void tree_open_many(const DeviceTree& tree, const uint64_t* d_indices, uint32_t count, uint32_t* d_out,
                    cudaStream_t st);

// Row leaves of C columns x 2^log_n M31 values (column c at d_cols + c * col_stride):
// leaf r = hashM31s(col_0[r], ..., col_{C-1}[r]) (src/m31/hash.zig:15-25), C <= 256.
// Also writes g[r] = sum_c gammas[c] * col_c[r] when `g_out` is not null, and, when
// `g_tree` is not null, the tree over hashQM31(g[r]).
void build_row_tree(const uint32_t* d_cols, size_t col_stride, uint32_t C, DeviceTree& tree, const qm31* d_gammas,
                    qm31* g_out, DeviceTree* g_tree, cudaStream_t st);
// The leaf level only of build_row_tree (and of the g tree); finish with tree_finish.
void build_row_leaves(const uint32_t* d_cols, size_t col_stride, uint32_t C, DeviceTree& tree, const qm31* d_gammas,
                      qm31* g_out, DeviceTree* g_tree, cudaStream_t st);

}  // namespace zs
