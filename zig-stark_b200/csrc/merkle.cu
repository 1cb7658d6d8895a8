// Merkle trees on the device (src/core/merkle/merkle.zig:17-68).
//
// Leaves and the first levels are built by one CTA per run of up to 256 leaves:
// each thread hashes its leaf with one Blake3 compression chain in registers, the
// CTA keeps the run's digests in shared memory and climbs its subtree (hash2 =
// Blake3("zig-stark:pair" || L || R), two compressions), writing every level
// because openings need them. Levels above the runs are finished by k_tree_up
// in the same way, 512 nodes per CTA.
#include "blake3.cuh"
#include "merkle.cuh"

namespace zs {

namespace {
constexpr unsigned kRun = 256;      // leaves per CTA in the leaf kernels
constexpr unsigned kSPad = kRun + 1;  // word-major digest rows in shared memory

// Climbs the subtree of `count` digests held word-major in d[w * kSPad + i],
// writing levels level0+1 .. level0+log2(count) of `tree`. `first` is the index
// (at level0) of the CTA's first digest.
__device__ void climb(uint32_t* d, unsigned count, uint32_t* tree_words, unsigned log_n, unsigned level0,
                      uint64_t first) {
  const size_t N2 = (size_t)2 << log_n;
  unsigned lvl = level0;
  for (unsigned cnt = count >> 1; cnt >= 1; cnt >>= 1) {
    ++lvl;
    const unsigned t = threadIdx.x;
    uint32_t o[8];
    const bool act = t < cnt;
    if (act) {
      uint32_t l[8], r[8];
#pragma unroll
      for (int w = 0; w < 8; ++w) {
        l[w] = d[w * kSPad + 2 * t];
        r[w] = d[w * kSPad + 2 * t + 1];
      }
      b3::hash2(l, r, o);
    }
    __syncthreads();
    if (act) {
#pragma unroll
      for (int w = 0; w < 8; ++w) d[w * kSPad + t] = o[w];
      const uint64_t idx = (first >> (lvl - level0)) + t;
      uint4* dst = reinterpret_cast<uint4*>(tree_words + 8 * (N2 - (N2 >> lvl) + idx));
      dst[0] = make_uint4(o[0], o[1], o[2], o[3]);
      dst[1] = make_uint4(o[4], o[5], o[6], o[7]);
    }
    __syncthreads();
  }
}

__device__ __forceinline__ void put_digest(uint32_t* tree_words, size_t digest_index, const uint32_t o[8]) {
  uint4* dst = reinterpret_cast<uint4*>(tree_words + 8 * digest_index);
  dst[0] = make_uint4(o[0], o[1], o[2], o[3]);
  dst[1] = make_uint4(o[4], o[5], o[6], o[7]);
}
}  // namespace

// hashQM31 leaves + subtree per CTA.
__global__ void __launch_bounds__(kRun) k_qm31_leaves(const qm31* __restrict__ vals, uint32_t* tree_words,
                                                      unsigned log_n) {
  __shared__ uint32_t d[8 * kSPad];
  const uint64_t first = (uint64_t)blockIdx.x * blockDim.x;
  const uint64_t i = first + threadIdx.x;
  const uint4 raw = __ldg(reinterpret_cast<const uint4*>(vals) + i);
  uint32_t o[8];
  b3::hash_qm31(qmake(raw.x, raw.y, raw.z, raw.w), o);
  put_digest(tree_words, i, o);
#pragma unroll
  for (int w = 0; w < 8; ++w) d[w * kSPad + threadIdx.x] = o[w];
  __syncthreads();
  climb(d, blockDim.x, tree_words, log_n, 0, first);
}

// Row leaves over C columns (+ optional gamma combination and its QM31 tree).
__global__ void __launch_bounds__(kRun) k_row_leaves(const uint32_t* __restrict__ cols, size_t col_stride,
                                                     uint32_t C, uint32_t* tree_words, unsigned log_n,
                                                     const qm31* __restrict__ gammas, qm31* g_out,
                                                     uint32_t* g_tree_words) {
  __shared__ uint32_t d[8 * kSPad];
  __shared__ qm31 sg[256];
  const bool comb = gammas != nullptr;
  if (comb)
    for (uint32_t c = threadIdx.x; c < C; c += blockDim.x) sg[c] = gammas[c];
  __syncthreads();
  const uint64_t first = (uint64_t)blockIdx.x * blockDim.x;
  const uint64_t r = first + threadIdx.x;
  qm31 acc = qzero();
  uint32_t cv[8];
  b3::iv(cv);
  const uint32_t nblocks = (C * 4 + 63) / 64 == 0 ? 1 : (C * 4 + 63) / 64;
  for (uint32_t blk = 0; blk < nblocks; ++blk) {
    uint32_t m[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const uint32_t w = blk * 16 + k;
      uint32_t v = 0;
      if (w < C) {
        v = __ldg(cols + (size_t)w * col_stride + r);
        if (comb) acc = qadd(acc, qmul_m(sg[w], v));
      }
      m[k] = v;
    }
    const int rem = (int)(C * 4) - (int)(blk * 64);
    const uint32_t len = rem >= 64 ? 64u : (uint32_t)rem;
    const uint32_t flags = (blk == 0 ? b3::CHUNK_START : 0u) | (blk == nblocks - 1 ? (b3::CHUNK_END | b3::ROOT) : 0u);
    b3::compress_cv(cv, m, len, flags);
  }
  put_digest(tree_words, r, cv);
#pragma unroll
  for (int w = 0; w < 8; ++w) d[w * kSPad + threadIdx.x] = cv[w];
  __syncthreads();
  climb(d, blockDim.x, tree_words, log_n, 0, first);
  if (!comb) return;
  if (g_out) reinterpret_cast<uint4*>(g_out)[r] = make_uint4(acc.a.a, acc.a.b, acc.b.a, acc.b.b);
  if (g_tree_words) {
    uint32_t o[8];
    b3::hash_qm31(acc, o);
    put_digest(g_tree_words, r, o);
#pragma unroll
    for (int w = 0; w < 8; ++w) d[w * kSPad + threadIdx.x] = o[w];
    __syncthreads();
    climb(d, blockDim.x, g_tree_words, log_n, 0, first);
  }
}

// Levels above `level0`: each CTA climbs from up to 2 * blockDim.x digests.
__global__ void __launch_bounds__(kRun) k_tree_up(uint32_t* tree_words, unsigned log_n, unsigned level0) {
  __shared__ uint32_t d[8 * kSPad];
  const size_t N2 = (size_t)2 << log_n;
  const uint64_t count_in = (uint64_t)1 << (log_n - level0);
  const unsigned per = 2 * blockDim.x < count_in ? 2 * blockDim.x : (unsigned)count_in;
  const uint64_t first = (uint64_t)blockIdx.x * per;
  const uint32_t* src = tree_words + 8 * (N2 - (N2 >> level0));
  // first level: pairs from global
  const unsigned t = threadIdx.x;
  const unsigned cnt = per >> 1;
  uint32_t o[8];
  if (t < cnt) {
    uint32_t l[8], r[8];
    const uint4* a = reinterpret_cast<const uint4*>(src + 8 * (first + 2 * t));
    uint4 a0 = a[0], a1 = a[1], b0 = a[2], b1 = a[3];
    l[0] = a0.x; l[1] = a0.y; l[2] = a0.z; l[3] = a0.w; l[4] = a1.x; l[5] = a1.y; l[6] = a1.z; l[7] = a1.w;
    r[0] = b0.x; r[1] = b0.y; r[2] = b0.z; r[3] = b0.w; r[4] = b1.x; r[5] = b1.y; r[6] = b1.z; r[7] = b1.w;
    b3::hash2(l, r, o);
    put_digest(tree_words, (N2 - (N2 >> (level0 + 1))) + (first >> 1) + t, o);
#pragma unroll
    for (int w = 0; w < 8; ++w) d[w * kSPad + t] = o[w];
  }
  __syncthreads();
  climb(d, cnt, tree_words, log_n, level0 + 1, first >> 1);
}

static unsigned log2u(uint64_t x) {
  unsigned l = 0;
  while (((uint64_t)1 << l) < x) ++l;
  return l;
}

void tree_finish(DeviceTree& tree, unsigned from_level, cudaStream_t st) {
  unsigned lvl = from_level;
  while (lvl < tree.log_n) {
    const uint64_t count = (uint64_t)1 << (tree.log_n - lvl);  // digests at lvl
    const unsigned threads = count >= 2 * kRun ? kRun : (unsigned)(count / 2);
    const uint64_t per = 2 * (uint64_t)threads;
    k_tree_up<<<(unsigned)(count / per), threads, 0, st>>>(tree.words, tree.log_n, lvl);
    lvl += log2u(per);
  }
  ZS_CUDA(cudaGetLastError());
}

void build_qm31_tree(const qm31* d_values, DeviceTree& tree, cudaStream_t st) {
  const uint64_t n = (uint64_t)1 << tree.log_n;
  const unsigned threads = n >= kRun ? kRun : (unsigned)n;
  k_qm31_leaves<<<(unsigned)(n / threads), threads, 0, st>>>(d_values, tree.words, tree.log_n);
  ZS_CUDA(cudaGetLastError());
  tree_finish(tree, log2u(threads), st);
}

void build_row_tree(const uint32_t* d_cols, size_t col_stride, uint32_t C, DeviceTree& tree, const qm31* d_gammas,
                    qm31* g_out, DeviceTree* g_tree, cudaStream_t st) {
  if (C == 0 || C > 256) throw Error(ZS_EMALFORMED, "row leaves need 1..256 columns");
  const uint64_t n = (uint64_t)1 << tree.log_n;
  const unsigned threads = n >= kRun ? kRun : (unsigned)n;
  k_row_leaves<<<(unsigned)(n / threads), threads, 0, st>>>(d_cols, col_stride, C, tree.words, tree.log_n, d_gammas,
                                                            g_out, g_tree ? g_tree->words : nullptr);
  ZS_CUDA(cudaGetLastError());
  tree_finish(tree, log2u(threads), st);
  if (g_tree) tree_finish(*g_tree, log2u(threads), st);
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
