// Merkle trees on the device (src/core/merkle/merkle.zig:17-68).
//
// Two kinds of kernels, both without block-wide barriers so every lane stays busy:
//   leaf kernels: one thread per leaf, one Blake3 compression chain in registers
//     (hashQM31 = 1 compression, hashM31s of a 64-value row = 4);
//   k_tree_up: one thread per 2^s consecutive digests of a level (s <= 3) folds them
//     into its own s-level subtree with hash2 (= Blake3("zig-stark:pair" || L || R),
//     two compressions), writing every node, because openings need all levels.
// A tree over 2^22 leaves therefore takes one leaf launch and eight tree launches.
#include <algorithm>

#include "blake3.cuh"
#include "merkle.cuh"

namespace zs {

namespace {
constexpr unsigned kThreads = 256;

__device__ __forceinline__ void put_digest(uint32_t* tree_words, size_t digest_index, const uint32_t o[8]) {
  uint4* dst = reinterpret_cast<uint4*>(tree_words + 8 * digest_index);
  dst[0] = make_uint4(o[0], o[1], o[2], o[3]);
  dst[1] = make_uint4(o[4], o[5], o[6], o[7]);
}
__device__ __forceinline__ void get_digest(const uint32_t* tree_words, size_t digest_index, uint32_t o[8]) {
  const uint4* src = reinterpret_cast<const uint4*>(tree_words + 8 * digest_index);
  const uint4 a = src[0], b = src[1];
  o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
  o[4] = b.x; o[5] = b.y; o[6] = b.z; o[7] = b.w;
}

// The subtree over CNT (2, 4 or 8) consecutive digests of `level0` starting at index
// `first` (a multiple of CNT): digests arrive in order from `next(k, d)`, a stack of
// pending left siblings merges them, and every new node is written.
template <int CNT, typename Next>
__device__ __forceinline__ void thread_subtree(Next&& next, uint32_t* tree_words, unsigned log_n, unsigned level0,
                                               uint64_t first) {
  const size_t N2 = (size_t)2 << log_n;
  uint32_t stk[3][8];
#pragma unroll
  for (int k = 0; k < CNT; ++k) {
    uint32_t cur[8];
    next(k, cur);
    int depth = __popc(k) ;  // pending left siblings before merging leaf k (k's set bits)
#pragma unroll
    for (int b = 0; (1 << (b + 1)) <= CNT; ++b) {
      if (((k >> b) & 1) == 0) break;
      --depth;
      uint32_t o[8];
      b3::hash2(stk[depth], cur, o);
#pragma unroll
      for (int w = 0; w < 8; ++w) cur[w] = o[w];
      const unsigned lvl = level0 + b + 1;
      put_digest(tree_words, (N2 - (N2 >> lvl)) + ((first + k) >> (b + 1)), cur);
    }
    if (k + 1 < CNT) {
#pragma unroll
      for (int w = 0; w < 8; ++w) stk[depth][w] = cur[w];
    }
  }
}
}  // namespace

// hashQM31 leaves (src/m31/hash.zig:33-37).
// blockIdx.y selects the tree of a set (its values `v_stride` elements after the previous).
__global__ void __launch_bounds__(kThreads) k_qm31_leaves(const qm31* __restrict__ vals, size_t v_stride,
                                                          TreeSet ts, uint64_t n) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint4 raw = __ldg(reinterpret_cast<const uint4*>(vals + blockIdx.y * v_stride) + i);
  uint32_t o[8];
  b3::hash_qm31(qmake(raw.x, raw.y, raw.z, raw.w), o);
  put_digest(ts.words[blockIdx.y], i, o);
}

// Row leaves hashM31s(col_0[r], ..., col_{C-1}[r]) (src/m31/hash.zig:15-25), and
// optionally g[r] = sum_c gammas[c] * col_c[r] with its hashQM31 leaf. The four
// coordinates of g accumulate unreduced 62-bit products in 64 bits (one wide
// multiply-add each) with a Mersenne fold every four columns: after a fold the
// accumulator is below 2^34, and four products below (p-1)^2 keep it below 2^64.
__device__ __forceinline__ uint64_t fold64(uint64_t x) { return (x & P) + (x >> 31); }
__device__ __forceinline__ uint32_t canon64(uint64_t x) {
  x = fold64(fold64(x));  // < 2^31 + 8
  const uint32_t s = (uint32_t)x;
  return umin32(s, s - P);
}

__global__ void __launch_bounds__(kThreads) k_row_leaves(const uint32_t* __restrict__ cols, size_t col_stride,
                                                         uint32_t C, uint32_t* tree_words, uint64_t n,
                                                         const qm31* __restrict__ gammas, qm31* g_out,
                                                         uint32_t* g_tree_words) {
  __shared__ uint4 sg[256];
  const bool comb = gammas != nullptr;
  if (comb)
    for (uint32_t c = threadIdx.x; c < C; c += blockDim.x) sg[c] = reinterpret_cast<const uint4*>(gammas)[c];
  __syncthreads();
  const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  uint64_t acc0 = 0, acc1 = 0, acc2 = 0, acc3 = 0;
  uint32_t cv[8];
  b3::iv(cv);
  const uint32_t nblocks = C * 4 <= 64 ? 1 : (C * 4 + 63) / 64;
  // The next block's 16 column loads are issued before the current block is
  // compressed, so their latency hides behind ~700 integer instructions.
  uint32_t nxt[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) nxt[k] = (uint32_t)k < C ? __ldg(cols + (size_t)k * col_stride + r) : 0u;
  for (uint32_t blk = 0; blk < nblocks; ++blk) {
    uint32_t m[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) m[k] = nxt[k];
    if (blk + 1 < nblocks) {
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const uint32_t w = (blk + 1) * 16 + k;
        nxt[k] = w < C ? __ldg(cols + (size_t)w * col_stride + r) : 0u;
      }
    }
    if (comb) {
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const uint32_t w = blk * 16 + k;
        if (w < C) {
          const uint4 g = sg[w];
          const uint32_t v = m[k];
          acc0 += (uint64_t)g.x * v;
          acc1 += (uint64_t)g.y * v;
          acc2 += (uint64_t)g.z * v;
          acc3 += (uint64_t)g.w * v;
        }
        if ((k & 3) == 3) {
          acc0 = fold64(acc0);
          acc1 = fold64(acc1);
          acc2 = fold64(acc2);
          acc3 = fold64(acc3);
        }
      }
    }
    const int rem = (int)(C * 4) - (int)(blk * 64);
    const uint32_t len = rem >= 64 ? 64u : (uint32_t)rem;
    const uint32_t flags = (blk == 0 ? b3::CHUNK_START : 0u) | (blk == nblocks - 1 ? (b3::CHUNK_END | b3::ROOT) : 0u);
    b3::compress_cv(cv, m, len, flags);
  }
  put_digest(tree_words, r, cv);
  if (!comb) return;
  const qm31 acc = qmake(canon64(acc0), canon64(acc1), canon64(acc2), canon64(acc3));
  if (g_out) reinterpret_cast<uint4*>(g_out)[r] = make_uint4(acc.a.a, acc.a.b, acc.b.a, acc.b.b);
  if (g_tree_words) {
    uint32_t o[8];
    b3::hash_qm31(acc, o);
    put_digest(g_tree_words, r, o);
  }
}

// Levels level0+1 .. level0+log2(CNT): thread t folds digests [t*CNT, (t+1)*CNT) of level0.
template <int CNT>
__global__ void __launch_bounds__(kThreads) k_tree_up(TreeSet ts, unsigned log_n, unsigned level0) {
  uint32_t* tree_words = ts.words[blockIdx.y];
  const uint64_t count = ((uint64_t)1 << (log_n - level0)) / CNT;
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  const size_t N2 = (size_t)2 << log_n;
  const uint32_t* src = tree_words + 8 * (N2 - (N2 >> level0));
  const uint64_t first = t * CNT;
  thread_subtree<CNT>([&](int k, uint32_t d[8]) { get_digest(src, first + k, d); }, tree_words, log_n, level0, first);
}

// Subtrees of a tree in CTAs: CTA b takes the 2^levels <= kTopMax digests
// [b 2^levels, (b + 1) 2^levels) of level `level0` and hashes the `levels` levels above
// them in shared memory, one node per thread, a barrier between levels. These levels
// are latency-bound (few nodes, each a chain of two compressions), so one launch
// replaces one launch per level; with levels = log_n - level0 one CTA finishes the tree.
constexpr unsigned kTopMax = 1024;
__global__ void __launch_bounds__(kTopMax / 2) k_tree_block(TreeSet ts, unsigned log_n, unsigned level0,
                                                            unsigned levels) {
  __shared__ uint32_t s[kTopMax][8];
  uint32_t* tree_words = ts.words[blockIdx.y];
  const size_t N2 = (size_t)2 << log_n;
  uint32_t cnt = 1u << levels;
  const uint32_t first = blockIdx.x << levels;  // first digest of this CTA at level0
  const uint32_t* src = tree_words + 8 * (N2 - (N2 >> level0));
  for (uint32_t i = threadIdx.x; i < cnt; i += blockDim.x) get_digest(src, first + i, s[i]);
  __syncthreads();
  for (unsigned lvl = level0 + 1; lvl <= level0 + levels; ++lvl) {
    cnt >>= 1;
    uint32_t o[8];
    const bool active = threadIdx.x < cnt;
    if (active) {
      b3::hash2(s[2 * threadIdx.x], s[2 * threadIdx.x + 1], o);
      put_digest(tree_words, (N2 - (N2 >> lvl)) + (first >> (lvl - level0)) + threadIdx.x, o);
    }
    __syncthreads();  // every child is read before a parent overwrites it
    if (active)
      for (int w = 0; w < 8; ++w) s[threadIdx.x][w] = o[w];
    __syncthreads();
  }
}

static unsigned log2u(uint64_t x) {
  unsigned l = 0;
  while (((uint64_t)1 << l) < x) ++l;
  return l;
}

static void launch_up(const TreeSet& ts, uint32_t count, unsigned log_n, unsigned lvl, unsigned s,
                      cudaStream_t st) {
  const uint64_t threads_total = ((uint64_t)1 << (log_n - lvl)) >> s;
  const dim3 grid((unsigned)((threads_total + kThreads - 1) / kThreads), count);
  switch (s) {
    case 1: k_tree_up<2><<<grid, kThreads, 0, st>>>(ts, log_n, lvl); break;
    case 2: k_tree_up<4><<<grid, kThreads, 0, st>>>(ts, log_n, lvl); break;
    default: k_tree_up<8><<<grid, kThreads, 0, st>>>(ts, log_n, lvl); break;
  }
}

// Three levels per launch while a level still gives every SM plenty of threads
// (one thread chains 7 nodes = 14 compressions); above that one level per launch,
// so the narrow top of the tree costs one hash2 of latency per level.
static unsigned levels_per_launch(unsigned log_n, unsigned lvl) {
  const unsigned remaining = log_n - lvl;
  if (remaining >= 3 && remaining >= 3 + 15) return 3;  // >= 2^15 threads of 8-node subtrees
  return 1;
}

static void finish_set(const TreeSet& ts, uint32_t count, unsigned log_n, unsigned from_level, cudaStream_t st) {
  unsigned lvl = from_level;
  while (lvl < log_n) {
    const unsigned rem = log_n - lvl;
    if (levels_per_launch(log_n, lvl) == 3) {  // wide levels: subtrees per thread
      launch_up(ts, count, log_n, lvl, 3, st);
      lvl += 3;
      continue;
    }
    const unsigned levels = rem < 10 ? rem : 10;  // narrow levels: subtrees per CTA
    k_tree_block<<<dim3(1u << (rem - levels), count), kTopMax / 2, 0, st>>>(ts, log_n, lvl, levels);
    lvl += levels;
  }
  ZS_CUDA(cudaGetLastError());
}

static TreeSet single(const DeviceTree& tree) {
  TreeSet ts{};
  ts.words[0] = tree.words;
  return ts;
}

void tree_finish(DeviceTree& tree, unsigned from_level, cudaStream_t st) {
  finish_set(single(tree), 1, tree.log_n, from_level, st);
}

uint32_t tree_finish_launches(unsigned log_n, unsigned from_level) {
  uint32_t k = 0;
  for (unsigned lvl = from_level; lvl < log_n; ++k) {
    const unsigned rem = log_n - lvl;
    lvl += levels_per_launch(log_n, lvl) == 3 ? 3 : (rem < 10 ? rem : 10);
  }
  return k;
}

void build_qm31_tree(const qm31* d_values, DeviceTree& tree, cudaStream_t st) {
  build_qm31_leaves(d_values, tree, st);
  tree_finish(tree, 0, st);
}

void build_qm31_leaves(const qm31* d_values, DeviceTree& tree, cudaStream_t st) {
  const uint64_t n = (uint64_t)1 << tree.log_n;
  k_qm31_leaves<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, st>>>(d_values, 0, single(tree), n);
  ZS_CUDA(cudaGetLastError());
}

void build_qm31_trees(const qm31* d_values, size_t v_stride, DeviceTree* const* trees, uint32_t count,
                      cudaStream_t st) {
  for (uint32_t t0 = 0; t0 < count; t0 += kTreeBatch) {
    const uint32_t c = std::min<uint32_t>(kTreeBatch, count - t0);
    const unsigned log_n = trees[t0]->log_n;
    TreeSet ts{};
    for (uint32_t k = 0; k < c; ++k) {
      if (trees[t0 + k]->log_n != log_n) throw Error(ZS_EGENERIC, "build_qm31_trees: trees of different sizes");
      ts.words[k] = trees[t0 + k]->words;
    }
    const uint64_t n = (uint64_t)1 << log_n;
    k_qm31_leaves<<<dim3((unsigned)((n + kThreads - 1) / kThreads), c), kThreads, 0, st>>>(
        d_values + (size_t)t0 * v_stride, v_stride, ts, n);
    ZS_CUDA(cudaGetLastError());
    finish_set(ts, c, log_n, 0, st);
  }
}

void build_row_leaves(const uint32_t* d_cols, size_t col_stride, uint32_t C, DeviceTree& tree, const qm31* d_gammas,
                      qm31* g_out, DeviceTree* g_tree, cudaStream_t st) {
  if (C == 0 || C > 256) throw Error(ZS_EMALFORMED, "row leaves need 1..256 columns");
  const uint64_t n = (uint64_t)1 << tree.log_n;
  k_row_leaves<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, st>>>(
      d_cols, col_stride, C, tree.words, n, d_gammas, g_out, g_tree ? g_tree->words : nullptr);
  ZS_CUDA(cudaGetLastError());
}

void build_row_tree(const uint32_t* d_cols, size_t col_stride, uint32_t C, DeviceTree& tree, const qm31* d_gammas,
                    qm31* g_out, DeviceTree* g_tree, cudaStream_t st) {
  if (C == 0 || C > 256) throw Error(ZS_EMALFORMED, "row leaves need 1..256 columns");
  const uint64_t n = (uint64_t)1 << tree.log_n;
  k_row_leaves<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, st>>>(
      d_cols, col_stride, C, tree.words, n, d_gammas, g_out, g_tree ? g_tree->words : nullptr);
  ZS_CUDA(cudaGetLastError());
  tree_finish(tree, 0, st);
  if (g_tree) tree_finish(*g_tree, 0, st);
}

// out[q * log_n * 8 ...] = siblings of indices[q], bottom-up.
__global__ void k_open_many(const uint32_t* tree_words, unsigned log_n, const uint64_t* indices, uint32_t count,
                            uint32_t* out) {
  const uint32_t q = blockIdx.x;
  if (q >= count) return;
  const size_t N2 = (size_t)2 << log_n;
  uint64_t idx = indices[q];
  for (unsigned lvl = threadIdx.x; lvl < log_n; lvl += blockDim.x) {
    const uint64_t sib = (idx >> lvl) ^ 1;
    const uint32_t* s = tree_words + 8 * (N2 - (N2 >> lvl) + sib);
    uint32_t* o = out + ((size_t)q * log_n + lvl) * 8;
#pragma unroll
    for (int w = 0; w < 8; ++w) o[w] = s[w];
  }
}

void tree_open_many(const DeviceTree& tree, const uint64_t* d_indices, uint32_t count, uint32_t* d_out,
                    cudaStream_t st) {
  if (count == 0 || tree.log_n == 0) return;
  k_open_many<<<count, 32, 0, st>>>(tree.words, tree.log_n, d_indices, count, d_out);
  ZS_CUDA(cudaGetLastError());
}

void tree_open_host(const DeviceTree& tree, uint64_t index, uint8_t* out, cudaStream_t st) {
  for (unsigned lvl = 0; lvl < tree.log_n; ++lvl) {
    const uint64_t sib = (index >> lvl) ^ 1;
    ZS_CUDA(cudaMemcpyAsync(out + 32 * lvl, tree.level(lvl) + 8 * sib, 32, cudaMemcpyDeviceToHost, st));
  }
  ZS_CUDA(cudaStreamSynchronize(st));
}

}  // namespace zs
