// FRI fold over QM31 fused with the commitment of the folded layer.
//
// fri.zig:209-219 folds y0 = L[j], y1 = L[j + n/2] at x = D_i[j] into
//   (y0 + y1) * inv2 + alpha * ((y0 - y1) * x^-1 * inv2).
// x^-1 is rebuilt from tables instead of a per-point inversion: D_i[j] is a unit of
// the QM31 ring, so its inverse is unique and equals
// (FRI_OFFSET^(2^i))^-1 * w_0^-(j * 2^i), w_0 = primitiveRootOfUnity(dlog). inv2 = 2^30.
#include "blake3.cuh"
#include "fri.cuh"
#include "host.cuh"

namespace zs {

__global__ void k_fold_tables(qm31 w0inv, qm31* tabs) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= 3 * 2048) return;
  const uint32_t which = k / 2048, e = k % 2048;
  // w0inv^(e * 2^(11 * which))
  qm31 base = w0inv;
  for (uint32_t s = 0; s < 11 * which; ++s) base = qmul(base, base);
  tabs[k] = qpow(base, e);
}

FoldTables::FoldTables(unsigned d, cudaStream_t s) : dlog(d), st(s) {
  if (dlog > 32) throw Error(ZS_EMALFORMED, "FRI domain log size above 32");
  ZS_CUDA(cudaMallocAsync(&tables, 3 * 2048 * sizeof(qm31), st));
  const qm31 w0 = q_root_of_unity(dlog);
  k_fold_tables<<<(3 * 2048 + 255) / 256, 256, 0, st>>>(qinv(w0), tables);
  ZS_CUDA(cudaGetLastError());
}
FoldTables::~FoldTables() { cudaFreeAsync(tables, st); }

qm31 FoldTables::offset_inv(unsigned layer) const { return qinv(qpow(q_fri_offset(), (uint64_t)1 << layer)); }

namespace {
constexpr unsigned kThreads = 256;
}  // namespace

__device__ __forceinline__ qm31 ld_q(const qm31* p) {
  const uint4 r = __ldg(reinterpret_cast<const uint4*>(p));
  return qmake(r.x, r.y, r.z, r.w);
}

// One fold output per thread, plus its hashQM31 leaf when the folded layer is committed.
__global__ void __launch_bounds__(kThreads) k_fold(const qm31* __restrict__ in, qm31* __restrict__ out, uint32_t half,
                                                   qm31 alpha, const qm31* __restrict__ alpha_dev, qm31 off_inv,
                                                   unsigned layer, const qm31* __restrict__ tabs,
                                                   uint32_t* leaf_words) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= half) return;
  if (alpha_dev) alpha = ld_q(alpha_dev);
  const qm31 y0 = ld_q(in + j), y1 = ld_q(in + j + half);
  const uint64_t k = (uint64_t)j << layer;
  qm31 xinv = qmul(ld_q(tabs + (k & 2047)), ld_q(tabs + 2048 + ((k >> 11) & 2047)));
  if (k >> 22) xinv = qmul(xinv, ld_q(tabs + 4096 + ((k >> 22) & 2047)));
  xinv = qmul(xinv, off_inv);
  constexpr uint32_t inv2 = 1u << 30;
  const qm31 hs = qmul_m(qadd(y0, y1), inv2);
  const qm31 hd = qmul_m(qmul(qsub(y0, y1), xinv), inv2);
  const qm31 r = qadd(hs, qmul(alpha, hd));
  reinterpret_cast<uint4*>(out)[j] = make_uint4(r.a.a, r.a.b, r.b.a, r.b.b);
  if (!leaf_words) return;
  uint32_t o[8];
  b3::hash_qm31(r, o);
  uint4* dst = reinterpret_cast<uint4*>(leaf_words + 8 * (size_t)j);
  dst[0] = make_uint4(o[0], o[1], o[2], o[3]);
  dst[1] = make_uint4(o[4], o[5], o[6], o[7]);
}

void fri_fold(const qm31* d_in, qm31* d_out, uint32_t half, const qm31& alpha, unsigned layer,
              const FoldTables& tabs, DeviceTree* next_tree, cudaStream_t st, bool finish_tree) {
  k_fold<<<(half + kThreads - 1) / kThreads, kThreads, 0, st>>>(d_in, d_out, half, alpha, nullptr,
                                                                tabs.offset_inv(layer), layer, tabs.tables,
                                                                next_tree ? next_tree->words : nullptr);
  ZS_CUDA(cudaGetLastError());
  if (next_tree && finish_tree) tree_finish(*next_tree, 0, st);
}

void fri_fold(const qm31* d_in, qm31* d_out, uint32_t half, const qm31* d_alpha, unsigned layer,
              const FoldTables& tabs, DeviceTree* next_tree, cudaStream_t st) {
  k_fold<<<(half + kThreads - 1) / kThreads, kThreads, 0, st>>>(d_in, d_out, half, qzero(), d_alpha,
                                                                tabs.offset_inv(layer), layer, tabs.tables,
                                                                next_tree ? next_tree->words : nullptr);
  ZS_CUDA(cudaGetLastError());
  if (next_tree) tree_finish(*next_tree, 0, st);
}

namespace {
__device__ __forceinline__ void put_dg(uint32_t* words, size_t index, const uint32_t o[8]) {
  uint4* dst = reinterpret_cast<uint4*>(words + 8 * index);
  dst[0] = make_uint4(o[0], o[1], o[2], o[3]);
  dst[1] = make_uint4(o[4], o[5], o[6], o[7]);
}
__device__ __forceinline__ void get_dg(const uint32_t* words, size_t index, uint32_t o[8]) {
  const uint4* src = reinterpret_cast<const uint4*>(words + 8 * index);
  const uint4 a = src[0], b = src[1];
  o[0] = a.x, o[1] = a.y, o[2] = a.z, o[3] = a.w, o[4] = b.x, o[5] = b.y, o[6] = b.z, o[7] = b.w;
}
}  // namespace

__global__ void __launch_bounds__(kTailMax / 4) k_fri_tail(const FriTail* __restrict__ ftp, Channel* ch) {
  const FriTail& ft = *ftp;
  __shared__ qm31 alpha_s;
  __shared__ __align__(16) unsigned char ch_raw[sizeof(Channel)];    // the transcript, for the CTA's life
  copy_state(ch_raw, ch, sizeof(Channel));
  Channel* chs = reinterpret_cast<Channel*>(ch_raw);
  __syncthreads();
  for (uint32_t c = 0; c < ft.count; ++c) {
    const unsigned lg = ft.log_size - c;
    const uint32_t size = 1u << lg;
    const qm31* in = ft.layer[c];
    uint32_t* tw = ft.tree[c];
    const size_t N2 = (size_t)2 << lg;
    // leaves and levels (merkle.zig:17-45), a barrier between levels
    for (uint32_t e = threadIdx.x; e < size; e += blockDim.x) {
      const uint4 r = *reinterpret_cast<const uint4*>(in + e);
      uint32_t o[8];
      b3::hash_qm31(qmake(r.x, r.y, r.z, r.w), o);
      put_dg(tw, e, o);
    }
    __syncthreads();
    for (unsigned lvl = 1; lvl <= lg; ++lvl) {
      const uint32_t nodes = size >> lvl;
      const uint32_t* below = tw + 8 * (N2 - (N2 >> (lvl - 1)));
      for (uint32_t e = threadIdx.x; e < nodes; e += blockDim.x) {
        uint32_t l[8], r[8], o[8];
        get_dg(below, 2 * e, l);
        get_dg(below, 2 * e + 1, r);
        b3::hash2(l, r, o);
        put_dg(tw, (N2 - (N2 >> lvl)) + e, o);
      }
      __syncthreads();
    }
    // transcript step (fri.zig:199-206): absorb the root, sample the challenge
    if (threadIdx.x == 0) {
      const uint32_t* root = tw + 8 * (N2 - 2);
      uint8_t b[32];
      for (int w = 0; w < 8; ++w) {
        ft.roots[8 * c + w] = root[w];
        for (int k = 0; k < 4; ++k) b[4 * w + k] = (uint8_t)(root[w] >> (8 * k));
      }
      chs->absorb_bytes(b, 32);
      alpha_s = chs->sample_q();
      ft.alphas[c] = alpha_s;
    }
    __syncthreads();
    // fold (fri.zig:209-219), as k_fold
    const qm31 alpha = alpha_s, off_inv = ft.off_inv[c];
    const unsigned layer = ft.first + c;
    const uint32_t half = size >> 1;
    qm31* out = ft.layer[c + 1];
    for (uint32_t j = threadIdx.x; j < half; j += blockDim.x) {
      const qm31 y0 = ld_q(in + j), y1 = ld_q(in + j + half);
      const uint64_t k = (uint64_t)j << layer;
      qm31 xinv = qmul(ld_q(ft.tables + (k & 2047)), ld_q(ft.tables + 2048 + ((k >> 11) & 2047)));
      if (k >> 22) xinv = qmul(xinv, ld_q(ft.tables + 4096 + ((k >> 22) & 2047)));
      xinv = qmul(xinv, off_inv);
      constexpr uint32_t inv2 = 1u << 30;
      const qm31 hs = qmul_m(qadd(y0, y1), inv2);
      const qm31 hd = qmul_m(qmul(qsub(y0, y1), xinv), inv2);
      const qm31 r = qadd(hs, qmul(alpha, hd));
      reinterpret_cast<uint4*>(out)[j] = make_uint4(r.a.a, r.a.b, r.b.a, r.b.b);
    }
    __syncthreads();
  }
  copy_state(ch, ch_raw, sizeof(Channel));
}

void fri_tail(const FriTail* ft, Channel* ch, cudaStream_t st) {
  k_fri_tail<<<1, kTailMax / 4, 0, st>>>(ft, ch);
  ZS_CUDA(cudaGetLastError());
}

}  // namespace zs
