// Circle FFT over M31 on the device: twiddle tables, the standalone forward and
// inverse transforms, and the fused low-degree extension (interpolate on the
// canonic trace domain, evaluate on the 2^B-times larger canonic domain).
//
// Reference semantics (src/m31/ntt/circle.zig):
//   circleFFT 195-246: interleave A/B, line layers i = lg-1 .. 1 (DIF, one twiddle
//     per block of 2^(i+1)), the circle layer i = 0, then bit-reverse.
//   circleIFFT 272-346: bit-reverse, circle layer, line layers 1 .. lg-1 with
//     inverted twiddles (ibutterfly), scale by 1/n, de-interleave.
//   Twiddles 65-106: the tree of bit-reversed x-coordinates of the halved cosets,
//     and the circle layer [y, -y, -x, x] derived from its first level.
//
// Device layout of a domain's twiddles (flat, n - 1 words used): the twiddle of
// block b at layer i is TW[n - (n >> i) + b]; layer 0 (the circle layer) occupies
// [0, n/2), layer i >= 1 the 2^(lg-1-i) words after it. The inverse table holds the
// elementwise M31 inverses. Both tables store each twiddle doubled (2t < 2^32), the
// form the butterflies' multiply takes (mmul2). Tables are generated on the device
// once per domain.
//
// Each transform is split into HBM passes over groups held in shared memory: the
// butterflies of layers [0, K) connect elements inside aligned runs of 2^K
// positions, layers [K, lg) connect elements that share the low K position bits.
// Inside a pass, each thread moves 2^r elements (r <= 5 layers) between shared
// memory and registers per chunk, so a pass costs one shared-memory round trip per
// five layers; for groups of 2^10 the chunks next to global memory load and store
// their registers directly, and shared memory carries only the transpose between them. Every butterfly is the reference's exact M31 butterfly with the
// reference's twiddle, so outputs are bit-identical.
#include "circle.cuh"

namespace zs {

// ---------------------------------------------------------------------------
// Twiddle tables
// ---------------------------------------------------------------------------

// Tree levels t = 0 .. lg-2: level t holds x(D^t(P_r)) for r < 2^(lg-2-t) in
// bit-reversed order, P_r = offset + r*step of the half coset (circle.zig:69-82).
__global__ void k_tw_tree(unsigned lg, cpoint offset, cpoint step, uint32_t* TW) {
  const uint32_t half = 1u << (lg - 1);
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= (1u << (lg - 2))) return;
  cpoint pt = padd(offset, pmul(step, r));
  for (unsigned t = 0; t + 2 <= lg; ++t) {
    if (r >= (1u << (lg - 2 - t))) break;
    const uint32_t off = half - (1u << (lg - 1 - t));
    TW[half + off + bitrev(r, lg - 2 - t)] = pt.x;
    pt = pdbl(pt);
  }
  if (r == 0) TW[2 * half - 1] = 1;  // the reference's padding slot
}

// Circle layer from the first tree level: (f0, f1) -> [f1, -f1, -f0, f0] (circle.zig:96-106).
__global__ void k_tw_circle_layer(unsigned lg, uint32_t* TW) {
  const uint32_t half = 1u << (lg - 1);
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (half >> 2)) return;
  const uint32_t f0 = TW[half + 2 * k], f1 = TW[half + 2 * k + 1];
  TW[4 * k] = f1;
  TW[4 * k + 1] = mneg(f1);
  TW[4 * k + 2] = mneg(f0);
  TW[4 * k + 3] = f0;
}

// lg = 1, 2: the reference's closed forms (circle.zig:210-220, 290-319) written as
// the same flat table: layer 0 = [y] or [y, -y], layer 1 = [x].
__global__ void k_tw_small(unsigned lg, cpoint p0, uint32_t* TW) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (lg == 1) {
    TW[0] = p0.y;
    TW[1] = 1;
  } else {
    TW[0] = p0.y;
    TW[1] = mneg(p0.y);
    TW[2] = p0.x;
    TW[3] = 1;
  }
}

// Inverse table, stored doubled like the forward one (see mmul2).
__global__ void k_invert(const uint32_t* in, uint32_t* out, uint32_t n) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) out[k] = minv(in[k]) << 1;
}

// Forward table doubled in place, after k_invert has read it.
__global__ void k_double(uint32_t* tw, uint32_t n) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) tw[k] <<= 1;
}

// canonicHalf(lg) (src/m31/circle/coset.zig:59-65): B = generator().neg(),
// offset = B * 2^(30-lg), step = B * 2^(32-lg).
void canonic_half(unsigned lg, cpoint* offset, cpoint* step) {
  const cpoint gen_neg = {1268011823u, mneg(2)};
  *offset = pmul(gen_neg, (uint64_t)1 << (30 - lg));
  *step = pmul(gen_neg, (uint64_t)1 << (32 - lg));
}

CircleDomain::CircleDomain(unsigned lg_, cudaStream_t st) : lg(lg_) {
  if (lg < 1 || lg > 28) throw Error(ZS_EMALFORMED, "circle domain log size must be in [1, 28]");
  cpoint offset, step;
  canonic_half(lg, &offset, &step);
  init(offset, step, st);
}

CircleDomain::CircleDomain(unsigned lg_, cpoint offset, cpoint step, cudaStream_t st) : lg(lg_) {
  if (lg < 1 || lg > 28) throw Error(ZS_EMALFORMED, "circle domain log size must be in [1, 28]");
  init(offset, step, st);
}

void CircleDomain::init(cpoint offset, cpoint step, cudaStream_t st) {
  const uint32_t n = 1u << lg;
  ZS_CUDA(cudaMallocAsync(&tw, n * sizeof(uint32_t), st));
  ZS_CUDA(cudaMallocAsync(&itw, n * sizeof(uint32_t), st));
  if (lg <= 2) {
    k_tw_small<<<1, 32, 0, st>>>(lg, offset, tw);
  } else {
    const uint32_t r = 1u << (lg - 2);
    k_tw_tree<<<(r + 255) / 256, 256, 0, st>>>(lg, offset, step, tw);
    const uint32_t k = 1u << (lg - 3);
    k_tw_circle_layer<<<(k + 255) / 256, 256, 0, st>>>(lg, tw);
  }
  k_invert<<<(n + 255) / 256, 256, 0, st>>>(tw, itw, n);
  k_double<<<(n + 255) / 256, 256, 0, st>>>(tw, n);
  ZS_CUDA(cudaGetLastError());
}

CircleDomain::~CircleDomain() {
  cudaFree(tw);
  cudaFree(itw);
}

// ---------------------------------------------------------------------------
// Butterfly arithmetic
// ---------------------------------------------------------------------------

// Every twiddle table of this file holds each twiddle doubled, t2 = 2t < 2^32. Then
// a * t2 = 2at, whose high word is at >> 31 and whose low word is 2 (at & p), so the
// Mersenne fold of at is hi + (lo >> 1) <= 2p - 2: one 32 x 32 -> 64 multiply and one
// shift-add, where a product of undoubled values needs a mask, a 64-bit shift and an
// add. The result is mmul's canonical value (field.cuh).
__device__ __forceinline__ uint32_t mmul2(uint32_t a, uint32_t t2) {
  const uint64_t prod = (uint64_t)a * t2;
  const uint32_t s = (uint32_t)(prod >> 32) + ((uint32_t)prod >> 1);
  return umin32(s, s - P);
}

// ---------------------------------------------------------------------------
// Shared-memory group transforms
// ---------------------------------------------------------------------------

// One padding word per 32 keeps strided chunk accesses on distinct banks.
__device__ __forceinline__ uint32_t padx(uint32_t e) { return e + (e >> 5); }
__host__ __device__ inline uint32_t group_stride(unsigned M) {
  const uint32_t g = 1u << M;
  return g + (g >> 5) + 1;
}

// Applies layers [b0, b0 + R) (group-local numbering; global layer = local + shift)
// to every group held in `s`. Element e of group gi sits at virtual position
// vb[gi] + e, so the twiddle of a butterfly at global layer i whose lower element
// has virtual position V is T_i[V >> (local layer + 1)].
template <int R, bool INV>
__device__ __forceinline__ void chunk(uint32_t* s, uint32_t gstride, unsigned G, unsigned M, unsigned b0,
                                      unsigned shift, const uint32_t* __restrict__ TW, uint32_t n_dom,
                                      const uint32_t* vb) {
  const unsigned sl = M - R;
  const uint32_t total = G << sl;
  for (uint32_t slot = threadIdx.x; slot < total; slot += blockDim.x) {
    const uint32_t gi = slot >> sl;
    const uint32_t rest = slot & ((1u << sl) - 1);
    const uint32_t e0 = ((rest >> b0) << (b0 + R)) | (rest & ((1u << b0) - 1));
    uint32_t* base = s + gi * gstride;
    uint32_t v[1 << R];
#pragma unroll
    for (int m = 0; m < (1 << R); ++m) v[m] = base[padx(e0 | ((uint32_t)m << b0))];
    const uint32_t Vh = (vb[gi] + e0) >> (b0 + R);
    if (!INV) {
#pragma unroll
      for (int l = R - 1; l >= 0; --l) {
        const unsigned i = b0 + l + shift;
        const uint32_t* T = TW + (n_dom - (n_dom >> i)) + (Vh << (R - l - 1));
        uint32_t tws[1 << (R - 1)];
#pragma unroll
        for (int hb = 0; hb < (1 << (R - 1)); ++hb)
          if (hb < (1 << (R - 1 - l))) tws[hb] = __ldg(T + hb);
#pragma unroll
        for (int m0 = 0; m0 < (1 << R); ++m0) {
          if (m0 & (1 << l)) continue;
          const int m1 = m0 | (1 << l);
          const uint32_t t = tws[m0 >> (l + 1)];
          const uint32_t x1 = mmul2(v[m1], t), x0 = v[m0];
          v[m1] = msub(x0, x1);
          v[m0] = madd(x0, x1);
        }
      }
    } else {
#pragma unroll
      for (int l = 0; l < R; ++l) {
        const unsigned i = b0 + l + shift;
        const uint32_t* T = TW + (n_dom - (n_dom >> i)) + (Vh << (R - l - 1));
        uint32_t tws[1 << (R - 1)];
#pragma unroll
        for (int hb = 0; hb < (1 << (R - 1)); ++hb)
          if (hb < (1 << (R - 1 - l))) tws[hb] = __ldg(T + hb);
#pragma unroll
        for (int m0 = 0; m0 < (1 << R); ++m0) {
          if (m0 & (1 << l)) continue;
          const int m1 = m0 | (1 << l);
          const uint32_t t = tws[m0 >> (l + 1)];
          const uint32_t x0 = v[m0], x1 = v[m1];
          v[m0] = madd(x0, x1);
          v[m1] = mmul2(msub(x0, x1), t);
        }
      }
    }
#pragma unroll
    for (int m = 0; m < (1 << R); ++m) base[padx(e0 | ((uint32_t)m << b0))] = v[m];
  }
}

template <bool INV>
__device__ __forceinline__ void chunk_dispatch(unsigned r, uint32_t* s, uint32_t gstride, unsigned G, unsigned M,
                                               unsigned b0, unsigned shift, const uint32_t* TW, uint32_t n_dom,
                                               const uint32_t* vb) {
  switch (r) {
    case 1: chunk<1, INV>(s, gstride, G, M, b0, shift, TW, n_dom, vb); break;
    case 2: chunk<2, INV>(s, gstride, G, M, b0, shift, TW, n_dom, vb); break;
    case 3: chunk<3, INV>(s, gstride, G, M, b0, shift, TW, n_dom, vb); break;
    default: chunk<4, INV>(s, gstride, G, M, b0, shift, TW, n_dom, vb); break;
  }
}

// C consecutive twiddles from T into registers, as 16- or 8-byte loads where C allows
// (a chunk's twiddle run for layer i starts at TW[n - (n >> i) + Vh * C], a multiple of
// C words from a 256-byte-aligned table, so the vector loads are aligned).
template <int C>
__device__ __forceinline__ void load_twiddles(uint32_t* dst, const uint32_t* __restrict__ T) {
  if constexpr (C >= 4) {
#pragma unroll
    for (int q = 0; q < C / 4; ++q) {
      const uint4 x = __ldg(reinterpret_cast<const uint4*>(T) + q);
      dst[4 * q] = x.x, dst[4 * q + 1] = x.y, dst[4 * q + 2] = x.z, dst[4 * q + 3] = x.w;
    }
  } else if constexpr (C == 2) {
    const uint2 x = __ldg(reinterpret_cast<const uint2*>(T));
    dst[0] = x.x, dst[1] = x.y;
  } else {
    dst[0] = __ldg(T);
  }
}

// The butterflies of local layer l of a chunk on the 2^R values in registers, with the
// layer's 2^(R-1-l) twiddles in tws.
template <int R, bool INV, int l>
__device__ __forceinline__ void layer_butterflies(uint32_t* v, const uint32_t* tws) {
#pragma unroll
  for (int m0 = 0; m0 < (1 << R); ++m0) {
    if (m0 & (1 << l)) continue;
    const int m1 = m0 | (1 << l);
    const uint32_t t = tws[m0 >> (l + 1)];
    if (!INV) {
      const uint32_t x1 = mmul2(v[m1], t), x0 = v[m0];
      v[m1] = msub(x0, x1);
      v[m0] = madd(x0, x1);
    } else {
      const uint32_t x0 = v[m0], x1 = v[m1];
      v[m0] = madd(x0, x1);
      v[m1] = mmul2(msub(x0, x1), t);
    }
  }
}

// The R layers of one chunk on the 2^R values in registers: layer LL of the chunk's
// order (top-down forward, bottom-up inverse), then the rest. base_i: the global layer
// of the chunk's lowest layer; Vh: the virtual block index of the slot's lowest
// element at the chunk's top.
template <int R, bool INV, int LL>
__device__ __forceinline__ void chunk_layers(uint32_t* v, const uint32_t* __restrict__ TW, uint32_t n_dom,
                                             unsigned base_i, uint32_t Vh) {
  if constexpr (LL < R) {
    constexpr int l = INV ? LL : R - 1 - LL;
    const unsigned i = base_i + l;
    uint32_t tws[1 << (R - 1 - l)];
    load_twiddles<(1 << (R - 1 - l))>(tws, TW + (n_dom - (n_dom >> i)) + (Vh << (R - l - 1)));
    layer_butterflies<R, INV, l>(v, tws);
    chunk_layers<R, INV, LL + 1>(v, TW, n_dom, base_i, Vh);
  }
}

// The circle layer (global layer 0) on 32 values in registers whose twiddles at layer 0
// start at block 16 Vh, with the first line layer's eight twiddles t1 = T_1[8 Vh ..]. A
// table of lg >= 3 holds at layer-0 entries 4k .. 4k + 3 the values f1, -f1, -f0, f0 of
// its layer-1 entries f0 = T_1[2k], f1 = T_1[2k + 1] (k_tw_circle_layer; the inverse
// table, elementwise inverses, keeps the pattern), so layer 0 needs no loads of its own:
// a butterfly with the negated twiddle swaps its two outputs (forward) or the operands
// of its subtraction (inverse), and gives the same canonical values.
template <bool INV>
__device__ __forceinline__ void circle_layer32(uint32_t* v, const uint32_t* t1) {
#pragma unroll
  for (int hb = 0; hb < 16; ++hb) {
    const int m0 = 2 * hb, m1 = m0 + 1, j = hb & 3;
    const uint32_t t = t1[2 * (hb >> 2) + (j < 2 ? 1 : 0)];
    const bool neg = j == 1 || j == 2;
    if (!INV) {
      const uint32_t y = mmul2(v[m1], t), x0 = v[m0];
      v[m1] = neg ? madd(x0, y) : msub(x0, y);
      v[m0] = neg ? msub(x0, y) : madd(x0, y);
    } else {
      const uint32_t x0 = v[m0], x1 = v[m1];
      v[m0] = madd(x0, x1);
      v[m1] = mmul2(neg ? msub(x1, x0) : msub(x0, x1), t);
    }
  }
}

// Global layers [0, 5) of a size-N transform (lg >= 3) on 32 values in registers whose
// top virtual block is Vh: chunk_layers<5, INV, 0>(v, TW, N, 0, Vh) with the circle
// layer's twiddles taken from the first line layer's.
template <bool INV>
__device__ __forceinline__ void low_chunk32(uint32_t* v, const uint32_t* __restrict__ TW, uint32_t N, uint32_t Vh) {
  uint32_t t1[8];
  load_twiddles<8>(t1, TW + (N >> 1) + (Vh << 3));
  if (INV) {
    circle_layer32<true>(v, t1);
    layer_butterflies<5, true, 1>(v, t1);
    uint32_t t2[4], t3[2], t4[1];
    load_twiddles<4>(t2, TW + (N - (N >> 2)) + (Vh << 2));
    layer_butterflies<5, true, 2>(v, t2);
    load_twiddles<2>(t3, TW + (N - (N >> 3)) + (Vh << 1));
    layer_butterflies<5, true, 3>(v, t3);
    load_twiddles<1>(t4, TW + (N - (N >> 4)) + Vh);
    layer_butterflies<5, true, 4>(v, t4);
  } else {
    uint32_t t2[4], t3[2], t4[1];
    load_twiddles<1>(t4, TW + (N - (N >> 4)) + Vh);
    layer_butterflies<5, false, 4>(v, t4);
    load_twiddles<2>(t3, TW + (N - (N >> 3)) + (Vh << 1));
    layer_butterflies<5, false, 3>(v, t3);
    load_twiddles<4>(t2, TW + (N - (N >> 2)) + (Vh << 2));
    layer_butterflies<5, false, 2>(v, t2);
    layer_butterflies<5, false, 1>(v, t1);
    circle_layer32<false>(v, t1);
  }
}

// Compile-time variant of `chunk` for a known group size 2^M and chunk offset B0.
// The chunk's index bits never overlap the slot's, so element m sits at
// padx(e0) + padx(m << B0): one runtime address per slot, immediate offsets after it.
// Reads the groups from `src` and writes them to `dst` (the same layout; in place when
// they are equal).
template <int R, bool INV, unsigned M, unsigned B0>
__device__ __forceinline__ void chunk_ct(const uint32_t* src, uint32_t* dst, uint32_t gstride, unsigned G,
                                         unsigned shift, const uint32_t* __restrict__ TW, uint32_t n_dom,
                                         const uint32_t* vb) {
  constexpr unsigned SL = M - R;
  const uint32_t total = G << SL;
  for (uint32_t slot = threadIdx.x; slot < total; slot += blockDim.x) {
    const uint32_t gi = slot >> SL;
    const uint32_t rest = slot & ((1u << SL) - 1);
    const uint32_t e0 = ((rest >> B0) << (B0 + R)) | (rest & ((1u << B0) - 1));
    const uint32_t off = gi * gstride + padx(e0);
    uint32_t v[1 << R];
#pragma unroll
    for (int m = 0; m < (1 << R); ++m) v[m] = src[off + (m << B0) + ((m << B0) >> 5)];
    const uint32_t Vh = (vb[gi] + e0) >> (B0 + R);
    chunk_layers<R, INV, 0>(v, TW, n_dom, B0 + shift, Vh);
#pragma unroll
    for (int m = 0; m < (1 << R); ++m) dst[off + (m << B0) + ((m << B0) >> 5)] = v[m];
  }
}

// All M layers with a compile-time chunk schedule (chunks of <= 5 layers, the
// largest first), DONE layers already applied. The first chunk reads `src`, every
// chunk writes `dst`.
template <bool INV, unsigned M, unsigned DONE>
__device__ __forceinline__ void run_layers_ct(const uint32_t* src, uint32_t* dst, uint32_t gstride, unsigned G,
                                              unsigned shift, const uint32_t* TW, uint32_t n_dom, const uint32_t* vb) {
  if constexpr (DONE < M) {
    constexpr unsigned REM = M - DONE;
    constexpr unsigned NCH = (REM + 4) / 5;
    constexpr unsigned R = (REM + NCH - 1) / NCH;
    // forward: top-down, the chunk covers [M - DONE - R, M - DONE); inverse: bottom-up
    constexpr unsigned B0 = INV ? DONE : M - DONE - R;
    chunk_ct<R, INV, M, B0>(src, dst, gstride, G, shift, TW, n_dom, vb);
    __syncthreads();
    run_layers_ct<INV, M, DONE + R>(dst, dst, gstride, G, shift, TW, n_dom, vb);
  }
}

// All M local layers: DIF top-down for the forward transform, DIT bottom-up for
// the inverse, in chunks of at most four layers.
template <bool INV>
__device__ __forceinline__ void run_layers(uint32_t* s, uint32_t gstride, unsigned G, unsigned M, unsigned shift,
                           const uint32_t* TW, uint32_t n_dom, const uint32_t* vb) {
  if (M == 0) return;
  switch (M) {
    case 8: return run_layers_ct<INV, 8, 0>(s, s, gstride, G, shift, TW, n_dom, vb);
    case 9: return run_layers_ct<INV, 9, 0>(s, s, gstride, G, shift, TW, n_dom, vb);
    case 10: return run_layers_ct<INV, 10, 0>(s, s, gstride, G, shift, TW, n_dom, vb);
    case 11: return run_layers_ct<INV, 11, 0>(s, s, gstride, G, shift, TW, n_dom, vb);
    default: break;
  }
  const unsigned nch = (M + 3) / 4, base = M / nch, extra = M % nch;
  if (!INV) {
    unsigned top = M;
    for (unsigned c = 0; c < nch; ++c) {
      const unsigned r = base + (c < extra ? 1 : 0);
      chunk_dispatch<false>(r, s, gstride, G, M, top - r, shift, TW, n_dom, vb);
      top -= r;
      __syncthreads();
    }
  } else {
    unsigned bot = 0;
    for (unsigned c = 0; c < nch; ++c) {
      const unsigned r = base + (c < extra ? 1 : 0);
      chunk_dispatch<true>(r, s, gstride, G, M, bot, shift, TW, n_dom, vb);
      bot += r;
      __syncthreads();
    }
  }
}

// ---------------------------------------------------------------------------
// Pass kernels. blockIdx.y = column; columns are `col_stride` words apart.
// ---------------------------------------------------------------------------

// 4-byte asynchronous global -> shared copies (LDGSTS): the copy of the next batch
// of groups runs while the current batch is transformed.
__device__ __forceinline__ void cp_async4(uint32_t* smem, const uint32_t* gmem) {
  const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// Bit reversal of a compile-time value (the unrolled loops' constant offsets).
__host__ __device__ constexpr uint32_t cbitrev(uint32_t x, unsigned bits) {
  uint32_t r = 0;
  for (unsigned b = 0; b < bits; ++b) r |= ((x >> b) & 1u) << (bits - 1 - b);
  return r;
}

constexpr unsigned kLowThreads = 256;

// Moves between global memory and a batch of G padded groups in shared memory, for a
// size-2^LG transform split at K (groups of 2^K), hb = LG - K. Two orders:
//   contiguous: element e of group t is global word gbase(t) + e;
//   bit-reversed: element bitrev_K(v) of group t is global word (v << hb) + g0 + t.
struct LowIO {
  // Calls f(smem offset, global offset) for every element of the bit-reversed order.
  template <typename F>
  __device__ __forceinline__ static void bitrev_order(unsigned K, unsigned G, unsigned hb, uint32_t g0, F&& f) {
    const unsigned lg_g = 31 - __clz(G);
    const uint32_t gstride = group_stride(K);
#pragma unroll 8
    for (uint32_t idx = threadIdx.x; idx < (G << K); idx += blockDim.x) {
      const uint32_t t = idx & (G - 1), v = idx >> lg_g;
      f(t * gstride + padx(bitrev(v, K)), ((size_t)v << hb) + g0 + t);
    }
  }

  // Calls f(smem offset, global offset) for every element of the contiguous order;
  // gbase(t) gives group t's first global word.
  template <typename B, typename F>
  __device__ __forceinline__ static void contiguous_order(unsigned K, unsigned G, B&& gbase, F&& f) {
    const uint32_t gsz = 1u << K, gstride = group_stride(K);
#pragma unroll 8
    for (uint32_t idx = threadIdx.x; idx < (G << K); idx += blockDim.x) {
      const uint32_t t = idx >> K, e = idx & (gsz - 1);
      f(t * gstride + padx(e), gbase(t) + e);
    }
  }
};

// The low pass of the inverse (INV) or forward transform over `iters` consecutive
// batches of G groups of 2^K elements per CTA (blockIdx.y = column), double-buffered:
// batch j + 1 is copied into shared memory while batch j is transformed and stored.
//   inverse: layers [0, K) of a size-2^LG transform; reads natural-order evaluations
//            through the reference's bit reversal, writes position order.
//   forward: layers [0, K) of a size-2^LG transform over contiguous groups, then the
//            reference's final bit reversal on the store (natural-order evaluations).
// Shared memory: two buffers of G padded groups, then two G-entry arrays of virtual
// group bases. Groups of 2^10 with G = 8 run k_low10 instead.
template <bool INV>
__global__ void __launch_bounds__(kLowThreads, 3) k_low(const uint32_t* __restrict__ src, size_t src_stride,
                                                     uint32_t* __restrict__ dst, size_t dst_stride, unsigned LG,
                                                     unsigned K_, unsigned G_, unsigned iters,
                                                     const uint32_t* __restrict__ TW) {
  extern __shared__ uint32_t sm[];
  using IO = LowIO;
  const unsigned K = K_, G = G_;
  const uint32_t N = 1u << LG, gstride = group_stride(K);
  const unsigned hb = LG - K;
  // buffer b at sm + b * G * gstride, its group bases at sm + 2 * G * gstride + b * G
  auto buf = [&](int b) { return sm + (uint32_t)b * G * gstride; };
  auto vbs = [&](int b) { return sm + 2 * G * gstride + (uint32_t)b * G; };
  const uint32_t* col = src + (size_t)blockIdx.y * src_stride;
  uint32_t* out = dst + (size_t)blockIdx.y * dst_stride;
  const uint32_t batch0 = blockIdx.x * iters;

  auto issue = [&](uint32_t j, int b) {
    const uint32_t g0 = (batch0 + j) * G;
    if (threadIdx.x < G) vbs(b)[threadIdx.x] = bitrev(g0 + threadIdx.x, hb) << K;
    uint32_t* s = buf(b);
    if (INV) {
      IO::bitrev_order(K, G, hb, g0, [&](uint32_t so, size_t go) { cp_async4(s + so, col + go); });
    } else {
      IO::contiguous_order(
          K, G, [&](uint32_t t) { return (size_t)bitrev(g0 + t, hb) << K; },
          [&](uint32_t so, size_t go) { cp_async4(s + so, col + go); });
    }
    cp_async_commit();
  };

  issue(0, 0);
  for (uint32_t j = 0; j < iters; ++j) {
    const int b = (int)(j & 1);
    if (j + 1 < iters)
      issue(j + 1, b ^ 1);
    else
      cp_async_commit();  // an empty group keeps "all but the newest group" meaning batch j
    cp_async_wait_one();
    __syncthreads();
    uint32_t* s = buf(b);
    const uint32_t* vb = vbs(b);
    const uint32_t g0 = (batch0 + j) * G;
    run_layers<INV>(s, gstride, G, K, 0, TW, N, vb);  // ends with a barrier
    if (INV) {
      IO::contiguous_order(
          K, G, [&](uint32_t t) { return (size_t)vb[t]; }, [&](uint32_t so, size_t go) { out[go] = s[so]; });
    } else {
      IO::bitrev_order(K, G, hb, g0, [&](uint32_t so, size_t go) { out[go] = s[so]; });
    }
    __syncthreads();  // buffer b is refilled by the next iteration's issue
  }
}

// Groups of 2^10 elements in two 5-layer chunks, 8 groups per batch, 256 threads. The
// chunks take two thread layouts over a batch:
//   strided:     group gs = tid / 32, r = tid % 32, elements r + 32 m;
//   consecutive: group gc = tid % 8,  r = tid / 8,  elements 32 r + m   (m < 32).
// The chunk next to a global-memory side moves its 32 values between registers and
// global memory directly, in the layout that keeps that side coalesced (strided for a
// contiguous group: 128-byte rows; consecutive for the bit-reversed order and the
// middle pass's interleaved groups: 8 groups' words side by side), so shared memory
// only carries the transpose between the two chunks. Groups sit kGS10 words apart;
// kGS10 = 4 (mod 32) and padx() put both layouts' 32 lanes on 32 distinct banks.
constexpr uint32_t kGS10 = 1060;
constexpr size_t kBatch10Words = 8 * kGS10;

__device__ __forceinline__ uint32_t* strided_at(uint32_t* s, uint32_t gs, uint32_t r) { return s + gs * kGS10 + r; }
__device__ __forceinline__ uint32_t* consecutive_at(uint32_t* s, uint32_t gc, uint32_t r) {
  return s + gc * kGS10 + 33 * r;
}

// k_low for K = 10, G = 8 (every size-2^LG transform with LG >= 13 that splits at 10):
// the same layers and orders, one barrier per batch, the batches alternating between two
// shared buffers (batch j + 2 overwrites batch j's buffer only after every thread has
// passed batch j + 1's barrier, so after batch j's reads). Each thread loads the next
// batch's 32 values into a second register array while it transforms the current one,
// so the global loads' latency is hidden behind a batch of arithmetic (two CTAs of 125
// registers per thread per SM instead of three of 80: measured faster).
template <bool INV>
__global__ void __launch_bounds__(kLowThreads, 2) k_low10(const uint32_t* __restrict__ src, size_t src_stride,
                                                        uint32_t* __restrict__ dst, size_t dst_stride, unsigned LG,
                                                        unsigned iters, const uint32_t* __restrict__ TW) {
  extern __shared__ uint32_t sm[];
  const uint32_t N = 1u << LG;
  const unsigned hb = LG - 10;
  const uint32_t* col = src + (size_t)blockIdx.y * src_stride;
  uint32_t* out = dst + (size_t)blockIdx.y * dst_stride;
  const uint32_t gs = threadIdx.x >> 5, rs = threadIdx.x & 31;
  const uint32_t gc = threadIdx.x & 7, rc = threadIdx.x >> 3;
  // element 32 rc + m of a group is bit-reversed row ((bitrev_5(m) << 5) | bitrev_5(rc))
  const size_t brc_row = (size_t)(__brev(rc) >> 27) << hb;
  uint32_t w[32];
  {
    const uint32_t g0 = blockIdx.x * iters * 8;
    if (!INV) {
      const uint32_t* gp = col + ((size_t)bitrev(g0 + gs, hb) << 10) + rs;
#pragma unroll
      for (int m = 0; m < 32; ++m) w[m] = __ldg(gp + 32 * m);
    } else {
      const uint32_t* gp = col + brc_row + g0 + gc;
#pragma unroll
      for (int m = 0; m < 32; ++m) w[m] = __ldg(gp + ((size_t)cbitrev(m, 5) << (hb + 5)));
    }
  }
  for (uint32_t j = 0; j < iters; ++j) {
    uint32_t* s = sm + (j & 1) * kBatch10Words;
    const uint32_t g0 = (blockIdx.x * iters + j) * 8;
    uint32_t v[32];
    if (!INV) {
      // layers [5, 10) on contiguous groups, then [0, 5), stored in bit-reversed order
      const uint32_t vs = bitrev(g0 + gs, hb);
#pragma unroll
      for (int m = 0; m < 32; ++m) v[m] = w[m];
      if (j + 1 < iters) {
        const uint32_t* gp = col + ((size_t)bitrev(g0 + 8 + gs, hb) << 10) + rs;
#pragma unroll
        for (int m = 0; m < 32; ++m) w[m] = __ldg(gp + 32 * m);
      }
      chunk_layers<5, false, 0>(v, TW, N, 5, vs);
      uint32_t* wp = strided_at(s, gs, rs);
#pragma unroll
      for (int m = 0; m < 32; ++m) wp[33 * m] = v[m];
      __syncthreads();
      const uint32_t* rp = consecutive_at(s, gc, rc);
#pragma unroll
      for (int m = 0; m < 32; ++m) v[m] = rp[m];
      low_chunk32<false>(v, TW, N, (bitrev(g0 + gc, hb) << 5) + rc);
      uint32_t* op = out + brc_row + g0 + gc;
#pragma unroll
      for (int m = 0; m < 32; ++m) op[(size_t)cbitrev(m, 5) << (hb + 5)] = v[m];
    } else {
      // layers [0, 5) read in bit-reversed order, then [5, 10), stored contiguous
#pragma unroll
      for (int m = 0; m < 32; ++m) v[m] = w[m];
      if (j + 1 < iters) {
        const uint32_t* gp = col + brc_row + g0 + 8 + gc;
#pragma unroll
        for (int m = 0; m < 32; ++m) w[m] = __ldg(gp + ((size_t)cbitrev(m, 5) << (hb + 5)));
      }
      low_chunk32<true>(v, TW, N, (bitrev(g0 + gc, hb) << 5) + rc);
      uint32_t* wp = consecutive_at(s, gc, rc);
#pragma unroll
      for (int m = 0; m < 32; ++m) wp[m] = v[m];
      __syncthreads();
      const uint32_t* rp = strided_at(s, gs, rs);
#pragma unroll
      for (int m = 0; m < 32; ++m) v[m] = rp[33 * m];
      const uint32_t vs = bitrev(g0 + gs, hb);
      chunk_layers<5, true, 0>(v, TW, N, 5, vs);
      uint32_t* op = out + ((size_t)vs << 10) + rs;
#pragma unroll
      for (int m = 0; m < 32; ++m) op[32 * m] = v[m];
    }
  }
}

// Middle pass over groups that share the low K position bits (M = L - K layers).
//   mode LDE:       inverse layers [K, L), scale 1/n, then for each of the 2^B
//                   quarters the forward layers [K, L) of the size-2^(L+B) transform
//                   (its top B layers only copy: the padded half is zero).
//   mode IFFT_ONLY: inverse layers [K, L), scale 1/n, store de-interleaved (A then B).
//   mode FFT_ONLY:  load A-then-B coefficients interleaved, forward layers [K, L).
enum MidMode : int { MID_LDE = 0, MID_IFFT_ONLY = 1, MID_FFT_ONLY = 2 };

constexpr unsigned kMidThreads = 256;

// Calls f(smem offset, global offset) for every element of k_mid's groups: element hi
// of group t (the groups share the low K position bits lo0 + t) is global word
// (hi << K) + lo0 + t. KC, MC, GC: 0, or K, M and G known at compile time with
// kMidThreads / G = 2^A and A <= 5 <= M; then hi = hlo + (k << A) for a per-thread hlo,
// padx(hi) = padx(hlo) + k (2^A + 2^A / 32) and every offset but the first is a constant.
template <unsigned KC, unsigned MC, unsigned GC, typename F>
__device__ __forceinline__ void mid_order(unsigned K, unsigned M, unsigned G, uint32_t lo0, F&& f) {
  if constexpr (KC != 0) {
    constexpr unsigned LG_G = 31 - __builtin_clz(GC), A = 31 - __builtin_clz(kMidThreads / GC);
    static_assert(A <= 5 && MC >= A, "fast middle-pass layout");
    const uint32_t t = threadIdx.x & (GC - 1), hlo = threadIdx.x >> LG_G;
    const uint32_t s0 = t * group_stride(MC) + padx(hlo);
    const size_t g0 = ((size_t)hlo << KC) + lo0 + t;
#pragma unroll
    for (uint32_t k = 0; k < (1u << (MC - A)); ++k)
      f(s0 + k * ((1u << A) + (1u << A) / 32), g0 + ((size_t)k << (A + KC)));
  } else {
    const unsigned lg_g = 31 - __clz(G);
    const uint32_t gstride = group_stride(M);
#pragma unroll 8
    for (uint32_t idx = threadIdx.x; idx < (G << M); idx += blockDim.x) {
      const uint32_t t = idx & (G - 1), hi = idx >> lg_g;
      f(t * gstride + padx(hi), ((size_t)hi << K) + lo0 + t);
    }
  }
}

// KC, MC, GC: the compile-time layout of mid_order (0, 0, 0: K, M and G at run time);
// 10, 10, 8 (the 2^20-row LDE) runs the LDE mode in the register-direct layouts of
// k_low10, with 1/n applied by the last inverse chunk.
template <unsigned KC = 0, unsigned MC = 0, unsigned GC = 0>
__global__ void __launch_bounds__(kMidThreads, 3) k_mid(const uint32_t* __restrict__ in, size_t in_stride,
                                                      uint32_t* __restrict__ out, size_t out_stride, unsigned L,
                                                      unsigned K_, unsigned B, unsigned G_,
                                                      const uint32_t* __restrict__ ITW_small,
                                                      const uint32_t* __restrict__ TW_big, int mode) {
  extern __shared__ uint32_t sm[];
  constexpr bool FAST = KC != 0;
  const unsigned K = FAST ? KC : K_, G = FAST ? GC : G_;
  const unsigned M = L - K;
  const uint32_t n = 1u << L, gstride = group_stride(M);
  uint32_t* s_in = sm;
  uint32_t* s_w = sm + G * gstride;
  uint32_t* vb = s_w + G * gstride;
  const uint32_t lo0 = blockIdx.x * G;
  const uint32_t* src = in + (size_t)blockIdx.y * in_stride;
  uint32_t* dst = out + (size_t)blockIdx.y * out_stride;
  if constexpr (FAST) {
    if (mode == MID_LDE && KC == 10 && MC == 10 && GC == 8) {
      // Two chunks per transform in the layouts of k_low10: the inverse's first chunk
      // reads global memory in the consecutive layout, its second chunk ends in the
      // strided layout, which is where each quarter's first forward chunk starts, so a
      // thread keeps its scaled inverse values in its own strided slots of s_in (no
      // barrier: only it reads them back); each quarter's second chunk writes global
      // memory from the consecutive layout. Element hi of group t is global word
      // (hi << 10) + lo0 + t.
      uint32_t* s_q = sm + kBatch10Words;
      const uint32_t gs = threadIdx.x >> 5, rs = threadIdx.x & 31;
      const uint32_t gc = threadIdx.x & 7, rc = threadIdx.x >> 3;
      const unsigned inv_n_shift = (31 - L) % 31;
      const size_t io = ((size_t)rc << 15) + lo0 + gc;  // hi = 32 rc + m
      uint32_t v[32];
#pragma unroll
      for (int m = 0; m < 32; ++m) v[m] = __ldg(src + io + ((size_t)m << 10));
      chunk_layers<5, true, 0>(v, ITW_small, n, 10, rc);
      uint32_t* cp = consecutive_at(s_in, gc, rc);
#pragma unroll
      for (int m = 0; m < 32; ++m) cp[m] = v[m];
      __syncthreads();
      uint32_t* sp = strided_at(s_in, gs, rs);
#pragma unroll
      for (int m = 0; m < 32; ++m) v[m] = sp[33 * m];
      chunk_layers<5, true, 0>(v, ITW_small, n, 15, 0);
#pragma unroll
      for (int m = 0; m < 32; ++m) sp[33 * m] = mshl(v[m], inv_n_shift);
      uint32_t* wq = strided_at(s_q, gs, rs);
      const uint32_t* rq = consecutive_at(s_q, gc, rc);
      for (uint32_t q = 0; q < (1u << B); ++q) {
#pragma unroll
        for (int m = 0; m < 32; ++m) v[m] = sp[33 * m];
        chunk_layers<5, false, 0>(v, TW_big, n << B, 15, q);
#pragma unroll
        for (int m = 0; m < 32; ++m) wq[33 * m] = v[m];
        __syncthreads();
#pragma unroll
        for (int m = 0; m < 32; ++m) v[m] = rq[m];
        chunk_layers<5, false, 0>(v, TW_big, n << B, 10, (q << 5) + rc);
        uint32_t* dq = dst + (size_t)q * n + io;
#pragma unroll
        for (int m = 0; m < 32; ++m) dq[(size_t)m << 10] = v[m];
        __syncthreads();  // s_q is rewritten by the next quarter
      }
      return;
    }
  }
  const unsigned lg_g = 31 - __clz(G);
  if (threadIdx.x < G) vb[threadIdx.x] = 0;
  if (mode == MID_FFT_ONLY) {
    // interleaved position p holds A[p/2] (even p) or B[p/2] (odd p)
    #pragma unroll 8
    for (uint32_t idx = threadIdx.x; idx < (G << M); idx += blockDim.x) {
      const uint32_t t = idx & (G - 1), hi = idx >> lg_g;
      const uint32_t p = (hi << K) | (lo0 + t);
      s_in[t * gstride + padx(hi)] = __ldg(src + ((p & 1) ? (n >> 1) + (p >> 1) : (p >> 1)));
    }
    __syncthreads();
    run_layers<false>(s_in, gstride, G, M, K, TW_big, n << B, vb);
    mid_order<0, 0, 0>(K, M, G, lo0, [&](uint32_t so, size_t go) { dst[go] = s_in[so]; });
    return;
  }
  mid_order<KC, MC, GC>(K, M, G, lo0, [&](uint32_t so, size_t go) { s_in[so] = __ldg(src + go); });
  __syncthreads();
  // 1/n = 2^(31 - L) mod p: scaling is a rotation of the 31-bit word.
  const unsigned inv_n_shift = (31 - L) % 31;
  if (mode == MID_IFFT_ONLY) {
    run_layers<true>(s_in, gstride, G, M, K, ITW_small, n, vb);
    #pragma unroll 8
    for (uint32_t idx = threadIdx.x; idx < (G << M); idx += blockDim.x) {
      const uint32_t t = idx & (G - 1), hi = idx >> lg_g;
      const uint32_t p = (hi << K) | (lo0 + t);
      const uint32_t v = mshl(s_in[t * gstride + padx(hi)], inv_n_shift);
      dst[(p & 1) ? (n >> 1) + (p >> 1) : (p >> 1)] = v;
    }
    return;
  }
  // the LDE with a run-time layout (the compile-time layout returned above)
  run_layers<true>(s_in, gstride, G, M, K, ITW_small, n, vb);
  mid_order<0, 0, 0>(K, M, G, lo0, [&](uint32_t so, size_t) { s_in[so] = mshl(s_in[so], inv_n_shift); });
  __syncthreads();
  for (uint32_t q = 0; q < (1u << B); ++q) {
    if (threadIdx.x < G) vb[threadIdx.x] = q << M;
    for (uint32_t idx = threadIdx.x; idx < G * gstride; idx += blockDim.x) s_w[idx] = s_in[idx];
    __syncthreads();
    run_layers<false>(s_w, gstride, G, M, K, TW_big, n << B, vb);
    uint32_t* dq = dst + (size_t)q * n;
    mid_order<0, 0, 0>(K, M, G, lo0, [&](uint32_t so, size_t go) { dq[go] = s_w[so]; });
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Host launch helpers
// ---------------------------------------------------------------------------

namespace {
constexpr uint32_t kGroupWords = 16384;  // words of group data per shared buffer

unsigned pick_split(unsigned L) {
  unsigned k = L <= 20 ? (L < 10 ? L : 10) : (L + 1) / 2;
  return k;
}
// Groups per CTA: up to `budget` words of group data per shared buffer, at most 16.
unsigned pick_groups(unsigned M, uint32_t n_groups, uint32_t budget = kGroupWords) {
  uint32_t g = budget >> M;
  if (g == 0) g = 1;
  if (g > 16) g = 16;
  if (g > n_groups) g = n_groups;
  return g;
}
size_t smem_bytes(unsigned M, unsigned G, unsigned buffers) {
  return ((size_t)buffers * G * group_stride(M) + G) * sizeof(uint32_t);
}
void set_smem(const void* fn, size_t bytes) {
  ZS_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}
// The low pass (k_low) over C columns of a size-2^LG transform split at K: batches of
// G groups (at most kLowWords words each), `iters` batches per CTA.
constexpr uint32_t kLowWords = 8192;
template <bool INV>
void launch_low(const uint32_t* src, size_t src_stride, uint32_t* dst, size_t dst_stride, uint32_t C, unsigned LG,
                unsigned K, const uint32_t* tw, cudaStream_t st) {
  const uint32_t ngroups = 1u << (LG - K);
  const unsigned G = pick_groups(K, ngroups, kLowWords);
  const uint32_t batches = ngroups / G;
  unsigned iters = 1;
  while (iters < 8 && batches % (iters * 2) == 0 && batches / (iters * 2) >= 16) iters *= 2;
  const size_t sb = ((size_t)2 * G * group_stride(K) + 2 * G) * sizeof(uint32_t);
  if (K == 10 && G == 8) {  // groups of 2^10 (every LG >= 13 split at 10): register-direct chunks
    const size_t sb10 = 2 * kBatch10Words * sizeof(uint32_t);
    set_smem((const void*)k_low10<INV>, sb10);
    k_low10<INV><<<dim3(batches / iters, C), kLowThreads, sb10, st>>>(src, src_stride, dst, dst_stride, LG, iters, tw);
  } else {
    set_smem((const void*)k_low<INV>, sb);
    k_low<INV><<<dim3(batches / iters, C), kLowThreads, sb, st>>>(src, src_stride, dst, dst_stride, LG, K, G, iters,
                                                                  tw);
  }
}
// The middle pass (k_mid) over C columns of a size-2^L transform split at K.
void launch_mid(const uint32_t* in, size_t in_stride, uint32_t* out, size_t out_stride, uint32_t C, unsigned L,
                unsigned K, unsigned B, const uint32_t* itw, const uint32_t* tw, int mode, cudaStream_t st) {
  const unsigned M = L - K;
  const uint32_t ngroups = 1u << K;
  const unsigned G = pick_groups(M, ngroups, kGroupWords / 2);
  size_t sb = smem_bytes(M, G, 2);
  const dim3 grid(ngroups / G, C);
  if (K == 10 && M == 10 && G == 8) {  // the 2^20 -> 2^22 LDE: compile-time layout
    sb = std::max(sb, 2 * kBatch10Words * sizeof(uint32_t));
    set_smem((const void*)k_mid<10, 10, 8>, sb);
    k_mid<10, 10, 8><<<grid, kMidThreads, sb, st>>>(in, in_stride, out, out_stride, L, K, B, G, itw, tw, mode);
  } else {
    set_smem((const void*)k_mid<>, sb);
    k_mid<><<<grid, kMidThreads, sb, st>>>(in, in_stride, out, out_stride, L, K, B, G, itw, tw, mode);
  }
}
}  // namespace

size_t lde_scratch_words(unsigned L, unsigned B, uint32_t C) {
  // tmp (C * 2^L) + mid (C * 2^(L+B))
  return (size_t)C * (((size_t)1 << L) + ((size_t)1 << (L + B)));
}

void circle_lde(const uint32_t* d_in, size_t in_stride, uint32_t* d_out, size_t out_stride, uint32_t C,
                unsigned L, unsigned B, const CircleDomain& small, const CircleDomain& big, uint32_t* scratch,
                cudaStream_t st) {
  if (small.lg != L || big.lg != L + B) throw Error(ZS_EGENERIC, "circle_lde: domain mismatch");
  const unsigned K = pick_split(L);
  const uint32_t n = 1u << L;
  uint32_t* tmp = scratch;
  uint32_t* mid = scratch + (size_t)C * n;
  launch_low<true>(d_in, in_stride, tmp, n, C, L, K, small.itw, st);
  launch_mid(tmp, n, mid, (size_t)n << B, C, L, K, B, small.itw, big.tw, MID_LDE, st);
  launch_low<false>(mid, (size_t)n << B, d_out, out_stride, C, L + B, K, big.tw, st);
  ZS_CUDA(cudaGetLastError());
}

void circle_fft(const uint32_t* d_coeffs, uint32_t* d_evals, uint32_t C, const CircleDomain& dom, uint32_t* scratch,
                cudaStream_t st) {
  const unsigned L = dom.lg, K = pick_split(L);
  const uint32_t n = 1u << L;
  launch_mid(d_coeffs, n, scratch, n, C, L, K, 0, dom.itw, dom.tw, MID_FFT_ONLY, st);
  launch_low<false>(scratch, n, d_evals, n, C, L, K, dom.tw, st);
  ZS_CUDA(cudaGetLastError());
}

void circle_ifft(const uint32_t* d_evals, uint32_t* d_coeffs, uint32_t C, const CircleDomain& dom, uint32_t* scratch,
                 cudaStream_t st) {
  const unsigned L = dom.lg, K = pick_split(L);
  const uint32_t n = 1u << L;
  launch_low<true>(d_evals, n, scratch, n, C, L, K, dom.itw, st);
  launch_mid(scratch, n, d_coeffs, n, C, L, K, 0, dom.itw, dom.tw, MID_IFFT_ONLY, st);
  ZS_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Table-parameterised variants for callers that own every buffer (the
// allocation-free entry point in noalloc.cu): the canonic domain's tables are
// written into caller memory, and the LDE takes the tables directly.
// ---------------------------------------------------------------------------

void circle_twiddles_into(unsigned lg, uint32_t* tw, uint32_t* itw, cudaStream_t st) {
  cpoint offset, step;
  canonic_half(lg, &offset, &step);
  const uint32_t n = 1u << lg;
  if (lg <= 2) {
    k_tw_small<<<1, 32, 0, st>>>(lg, offset, tw);
  } else {
    const uint32_t r = 1u << (lg - 2);
    k_tw_tree<<<(r + 255) / 256, 256, 0, st>>>(lg, offset, step, tw);
    const uint32_t k = 1u << (lg - 3);
    k_tw_circle_layer<<<(k + 255) / 256, 256, 0, st>>>(lg, tw);
  }
  k_invert<<<(n + 255) / 256, 256, 0, st>>>(tw, itw, n);
  k_double<<<(n + 255) / 256, 256, 0, st>>>(tw, n);
  ZS_CUDA(cudaGetLastError());
}

void circle_lde_tables(const uint32_t* d_in, size_t in_stride, uint32_t* d_out, size_t out_stride, uint32_t C,
                       unsigned L, unsigned B, const uint32_t* itw_small, const uint32_t* tw_big, uint32_t* scratch,
                       cudaStream_t st) {
  const unsigned K = pick_split(L);
  const uint32_t n = 1u << L;
  uint32_t* tmp = scratch;
  uint32_t* mid = scratch + (size_t)C * n;
  launch_low<true>(d_in, in_stride, tmp, n, C, L, K, itw_small, st);
  launch_mid(tmp, n, mid, (size_t)n << B, C, L, K, B, itw_small, tw_big, MID_LDE, st);
  launch_low<false>(mid, (size_t)n << B, d_out, out_stride, C, L + B, K, tw_big, st);
  ZS_CUDA(cudaGetLastError());
}

}  // namespace zs
