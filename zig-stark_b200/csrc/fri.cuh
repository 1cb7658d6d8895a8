// FRI folding over QM31 on the device (src/m31/fri.zig).
#pragma once
#include "merkle.cuh"

namespace zs {

// Inverse domain points of the FRI layers of a size-2^dlog domain
// (D_i[j] = FRI_OFFSET^(2^i) * w_{dlog-i}^j, fri.zig:96-117): w_0^-k is the
// product of three 2^11-entry tables, so any k < 2^33 costs two QM31 products.
struct FoldTables {
  unsigned dlog = 0;
  qm31* tables = nullptr;  // 3 * 2048 entries
  cudaStream_t st = nullptr;  // freed in stream order
  explicit FoldTables(unsigned dlog, cudaStream_t st);
  ~FoldTables();
  FoldTables(const FoldTables&) = delete;
  FoldTables& operator=(const FoldTables&) = delete;
  // (FRI_OFFSET^(2^layer))^-1, host-side.
  qm31 offset_inv(unsigned layer) const;
};

// One fold (fri.zig:209-219): out[j] = (y0 + y1)/2 + alpha * (y0 - y1) / (2 D_layer[j]),
// y0 = in[j], y1 = in[j + half], for j < half. When `next_tree` is given, also
// writes the leaves hashQM31(out[j]) and, unless `finish_tree` is false (the caller
// finishes it elsewhere), the rest of the folded layer's tree.
void fri_fold(const qm31* d_in, qm31* d_out, uint32_t half, const qm31& alpha, unsigned layer,
              const FoldTables& tabs, DeviceTree* next_tree, cudaStream_t st, bool finish_tree = true);
// The same fold with the challenge read from device memory (written there by the
// device transcript step that precedes it on `st`).
void fri_fold(const qm31* d_in, qm31* d_out, uint32_t half, const qm31* d_alpha, unsigned layer,
              const FoldTables& tabs, DeviceTree* next_tree, cudaStream_t st);

// The small layers of the commit phase in one CTA (fri.zig:195-227): for layers
// first .. first + count - 1 (the first holding at most kTailMax values): commit the
// layer (hashQM31 leaves and the whole tree), absorb its root into the device
// transcript `ch` and sample the folding challenge, fold into the next layer. Every
// step is a barrier apart, so the chain of small dependent steps costs no launches.
constexpr uint32_t kTailMax = 1024;
constexpr uint32_t kTailLayers = 16;
struct FriTail {
  uint32_t first, count;  // absolute index of the first layer, layers handled
  unsigned log_size;      // log2 of the first layer's length
  const qm31* tables;     // FoldTables::tables
  qm31 off_inv[kTailLayers];
  qm31* layer[kTailLayers + 1];  // layer[c] has 2^(log_size - c) values; the last is only written
  uint32_t* tree[kTailLayers];   // DeviceTree words of layer c
  uint32_t* roots;               // 8 words per handled layer
  qm31* alphas;                  // one per handled layer
};
struct Channel;
// Launch with one CTA of kTailMax / 4 threads; `ft` and `ch` are in device memory.
void fri_tail(const FriTail* ft, Channel* ch, cudaStream_t st);

}  // namespace zs
