// The Binius sum-check on the device: the values[t] hook of src/binius/accel.zig:9-47
// (computed in src/binius/sumcheck.zig:357-372, GPU-ported by src/cuda/kernels/sumcheck.cu
// and src/cuda/sumcheck_gpu.zig:36-151), the table fold of sumcheck.zig:379-388, and the
// combination prover of sumcheck.zig:208-395 with its tables resident in device memory.
//
//   values[t] = sum_{rest < half} sum_terms coeff * prod_{f in term} (a_f + t (a_f + b_f)),
//   a_f = cur[f][2 rest], b_f = cur[f][2 rest + 1], t = 0..dmax, in the tower field
//   TowerField(3) = GF(2^8) or TowerField(7) = GF(2^128) (src/binius/tower.zig), where
//   addition is XOR.
//
// Tower arithmetic. The product of two GF(2^8) elements comes from a 64 KB table held in
// each CTA's shared memory, built once per device by the Karatsuba recursion that defines
// the tower (tower.zig:192-212). Above GF(2^8) a product at level L is three products at
// level L - 1 and one product by the level's constant beta = X_(L-2), the adjoined root of
// level L - 1: for c = c0 + c1 X_(L-2), c X_(L-2) = c1 + (c0 + c1 beta') X_(L-2), so it
// costs one table lookup at any level. A GF(2^128) product is 81 + 40 lookups. The points
// t < 256 lie in the GF(2^8) subfield, and a subfield scalar multiplies the 16 byte
// coordinates of a GF(2^128) element independently (the tower is a GF(2^8)-vector space
// on the monomials of X_3..X_6); t = 0 and t = 1 need no product at all (a and b), and
// t = 2, 3 only bit operations (2 = X_0 scales each 2-bit GF(4) coordinate on its own).
//
// The round's term list (at most 256 terms and 1024 factor indices) travels as the
// kernel's parameter (7.2 KB, within the 32 KB parameter space of sm_70 and later), so a
// round needs no device copy of it.
//
// Reduction. Each thread accumulates its rows for every point in registers (up to eight
// points; beyond that one point per pass), a warp XOR-reduces with shuffles, each warp
// XORs its result into shared memory, and each CTA XORs its values into the output words:
// one atomic per CTA and word, where the reference kernel takes one per thread.
//
// Fold. next[f][rest] = a + r (a + b). Over GF(2^8) the product by r is one lookup in row r
// of the table. Over GF(2^128) the product by a fixed r is GF(2^8)-linear in the 16 byte
// coordinates of (a + b): a 16 x 256 table of r * (v X^byte k), built once per fold, turns
// it into 16 lookups of 16 bytes.
//
// Prover. The tables go to the device once; each round is the values kernel, k_sc_step
// (the coefficients from a Lagrange matrix built once per proof, then the SHA-256
// transcript step in one thread, the challenge left in device memory) and the fold, which
// reads the challenge there: the rounds run back to back and the host waits once.
#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include "../../include/zs_binius.h"
#include "common.cuh"

namespace zs {
namespace {

using u128 = unsigned __int128;

constexpr unsigned kBThreads = 256;
constexpr uint32_t kMaxTerms = 256, kMaxFactors = 1024, kMaxPoint = 255, kMaxTables = 65535;
constexpr uint32_t kProveMaxPoints = 64;  // sumcheck.zig:243 (dmax + 1 <= 64)
constexpr int kRegPoints = 8;             // dmax < kRegPoints: every point in registers

// ---- host: the GF(2^8) product table ---------------------------------------------

uint32_t tower_mul_small(unsigned level, uint32_t a, uint32_t b) {  // level <= 3
  if (level == 0) return a & b & 1u;
  const unsigned half = 1u << (level - 1);
  const uint32_t mask = (1u << half) - 1;
  const uint32_t a0 = a & mask, a1 = (a >> half) & mask, b0 = b & mask, b1 = (b >> half) & mask;
  const uint32_t c0 = tower_mul_small(level - 1, a0, b0), c1 = tower_mul_small(level - 1, a1, b1);
  const uint32_t c2 = tower_mul_small(level - 1, a0 ^ a1, b0 ^ b1);
  const uint32_t beta = level == 1 ? 1u : 1u << (1u << (level - 2));
  return (c0 ^ c1) | ((c2 ^ c0 ^ c1 ^ tower_mul_small(level - 1, c1, beta)) << half);
}

// ---- tower arithmetic over a GF(2^8) product table (host and device) ----------

struct g128 {
  uint64_t lo, hi;
};
ZS_HD g128 gxor(const g128& a, const g128& b) { return {a.lo ^ b.lo, a.hi ^ b.hi}; }

struct Tower {
  // T[(a << 8) | b] = a * b in GF(2^8): shared memory on the device. A constant operand
  // goes first: its row is fixed and the variable operand spreads the lanes of a warp
  // over the banks (a constant second operand puts every lane in one bank).
  const uint8_t* T;
  ZS_HD uint32_t m8(uint32_t a, uint32_t b) const { return T[(a << 8) | b]; }
  // x * X_3 at level 4 (x * 0x100), from x = e0 + e1 X_3: e1 + (e0 + e1 X_2) X_3
  ZS_HD uint32_t a16(uint32_t x) const {
    const uint32_t e0 = x & 0xff, e1 = x >> 8;
    return e1 | ((e0 ^ m8(0x10, e1)) << 8);
  }
  ZS_HD uint32_t m16(uint32_t a, uint32_t b) const {
    const uint32_t a0 = a & 0xff, a1 = a >> 8, b0 = b & 0xff, b1 = b >> 8;
    const uint32_t c0 = m8(a0, b0), c1 = m8(a1, b1), c2 = m8(a0 ^ a1, b0 ^ b1);
    return (c0 ^ c1) | ((c2 ^ c0 ^ c1 ^ m8(0x10, c1)) << 8);
  }
  ZS_HD uint32_t a32(uint32_t x) const {
    const uint32_t e0 = x & 0xffff, e1 = x >> 16;
    return e1 | ((e0 ^ a16(e1)) << 16);
  }
  ZS_HD uint32_t m32(uint32_t a, uint32_t b) const {
    const uint32_t a0 = a & 0xffff, a1 = a >> 16, b0 = b & 0xffff, b1 = b >> 16;
    const uint32_t c0 = m16(a0, b0), c1 = m16(a1, b1), c2 = m16(a0 ^ a1, b0 ^ b1);
    return (c0 ^ c1) | ((c2 ^ c0 ^ c1 ^ a16(c1)) << 16);
  }
  ZS_HD uint64_t a64(uint64_t x) const {
    const uint32_t e0 = (uint32_t)x, e1 = (uint32_t)(x >> 32);
    return (uint64_t)e1 | ((uint64_t)(e0 ^ a32(e1)) << 32);
  }
  ZS_HD uint64_t m64(uint64_t a, uint64_t b) const {
    const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32), b0 = (uint32_t)b, b1 = (uint32_t)(b >> 32);
    const uint32_t c0 = m32(a0, b0), c1 = m32(a1, b1), c2 = m32(a0 ^ a1, b0 ^ b1);
    return (uint64_t)(c0 ^ c1) | ((uint64_t)(c2 ^ c0 ^ c1 ^ a32(c1)) << 32);
  }
  // level 7: beta = X_5, the root of level 6
  ZS_HD g128 m128(const g128& a, const g128& b) const {
    const uint64_t c0 = m64(a.lo, b.lo), c1 = m64(a.hi, b.hi), c2 = m64(a.lo ^ a.hi, b.lo ^ b.hi);
    return {c0 ^ c1, c2 ^ c0 ^ c1 ^ a64(c1)};
  }
  // s * x for a GF(2^8) scalar s: every byte coordinate of x times s
  ZS_HD uint64_t s64(uint32_t s, uint64_t x) const {
    uint64_t r = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) r |= (uint64_t)m8(s, (uint32_t)(x >> (8 * k)) & 0xff) << (8 * k);
    return r;
  }
  ZS_HD g128 s128(uint32_t s, const g128& x) const { return {s64(s, x.lo), s64(s, x.hi)}; }
};

// Levels 3..7 on the host over the GF(2^8) product table; inverses by the norm to the subfield:
// for a = a0 + a1 y with y^2 = beta y + 1, a (a0 + a1 beta + a1 y) = a0^2 + a0 a1 beta + a1^2.
struct HostTower {
  std::vector<uint8_t> T, I;
  HostTower() : T(65536), I(256, 0) {
    for (uint32_t a = 0; a < 256; ++a)
      for (uint32_t b = 0; b < 256; ++b) {
        T[(a << 8) | b] = (uint8_t)tower_mul_small(3, a, b);
        if (T[(a << 8) | b] == 1) I[a] = (uint8_t)b;
      }
  }
  static u128 beta(unsigned level) { return (u128)1 << (1u << (level - 2)); }
  u128 mul(unsigned level, u128 a, u128 b) const {
    const Tower F{T.data()};
    switch (level) {
      case 3: return F.m8((uint32_t)a, (uint32_t)b);
      case 4: return F.m16((uint32_t)a, (uint32_t)b);
      case 5: return F.m32((uint32_t)a, (uint32_t)b);
      case 6: return F.m64((uint64_t)a, (uint64_t)b);
      default: {
        const g128 p = F.m128({(uint64_t)a, (uint64_t)(a >> 64)}, {(uint64_t)b, (uint64_t)(b >> 64)});
        return (u128)p.hi << 64 | p.lo;
      }
    }
  }
  u128 inv(unsigned level, u128 a) const {
    if (level == 3) return I[(uint32_t)a];
    const unsigned half = 1u << (level - 1);
    const u128 mask = ((u128)1 << half) - 1;
    const u128 a0 = a & mask, a1 = a >> half, bt = beta(level);
    const u128 lo = a0 ^ mul(level - 1, a1, bt);
    const u128 nrm = mul(level - 1, a0, lo) ^ mul(level - 1, a1, a1);
    const u128 ni = inv(level - 1, nrm);
    return mul(level - 1, lo, ni) | (mul(level - 1, a1, ni) << half);
  }
};

const HostTower& host_tower() {
  static const HostTower t;
  return t;
}

// ---- device: the product table and the kernels -----------------------------------

// One round's term list, passed by value: term k multiplies coefficient k (coef[es k ..];
// kind[k]: 0 = the unit, 1 = an element of the GF(2^8) subfield, 2 = any other) by its
// factor tables idx[off[k] .. off[k + 1]).
struct Terms {
  uint32_t nterms;
  uint32_t off[kMaxTerms + 1];
  uint16_t idx[kMaxFactors];
  uint8_t kind[kMaxTerms];
  alignas(16) uint8_t coef[16 * kMaxTerms];
};

__device__ __forceinline__ void load_table(uint8_t* s_T, const uint8_t* __restrict__ gT) {
  const uint4* src = reinterpret_cast<const uint4*>(gT);
  uint4* dst = reinterpret_cast<uint4*>(s_T);
  for (uint32_t k = threadIdx.x; k < 65536 / 16; k += blockDim.x) dst[k] = src[k];
}

// XOR of `v` over the warp into `acc` (shared memory).
__device__ __forceinline__ void warp_xor_into(uint32_t v, uint32_t* acc) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v ^= __shfl_xor_sync(0xffffffffu, v, d);
  if ((threadIdx.x & 31) == 0 && v) atomicXor(acc, v);
}

__device__ __forceinline__ void warp_xor_into128(const g128& v, uint32_t* acc) {
  warp_xor_into((uint32_t)v.lo, acc);
  warp_xor_into((uint32_t)(v.lo >> 32), acc + 1);
  warp_xor_into((uint32_t)v.hi, acc + 2);
  warp_xor_into((uint32_t)(v.hi >> 32), acc + 3);
}

// 2 x, by bits: 2 = X_0 lies in GF(4), and a GF(4) scalar scales each GF(4) coordinate (bit
// pair) of a tower element on its own: (a0, a1) -> a1 + (a0 + a1) X_0.
ZS_HD uint32_t mul2_8(uint32_t x) { return ((x >> 1) & 0x55u) | (((x << 1) ^ x) & 0xAAu); }
ZS_HD uint64_t mul2_64(uint64_t x) {
  return ((x >> 1) & 0x5555555555555555ull) | (((x << 1) ^ x) & 0xAAAAAAAAAAAAAAAAull);
}

// The point t's linear factor a + t (a + b): a at t = 0, b at t = 1, a + 2 (a + b) and
// b + 2 (a + b) at t = 2 and 3 (no table lookup), a lookup beyond.
template <int t>
__device__ __forceinline__ uint32_t at_point8(const Tower& F, uint32_t a, uint32_t b) {
  if constexpr (t == 0) return a;
  else if constexpr (t == 1) return b;
  else if constexpr (t == 2) return a ^ mul2_8(a ^ b);
  else if constexpr (t == 3) return b ^ mul2_8(a ^ b);
  else return a ^ F.m8(t, a ^ b);
}
template <int t>
__device__ __forceinline__ g128 at_point128(const Tower& F, const g128& a, const g128& b) {
  if constexpr (t == 0) return a;
  else if constexpr (t == 1) return b;
  else if constexpr (t == 2) return {a.lo ^ mul2_64(a.lo ^ b.lo), a.hi ^ mul2_64(a.hi ^ b.hi)};
  else if constexpr (t == 3) return {b.lo ^ mul2_64(a.lo ^ b.lo), b.hi ^ mul2_64(a.hi ^ b.hi)};
  else return gxor(a, F.s128(t, gxor(a, b)));
}

// prod[t] = (first factor at t), then prod[t] *= (next factor at t), for t < D.
template <int D, int t = 0>
__device__ __forceinline__ void first8(const Tower& F, uint32_t (&prod)[D], uint32_t a, uint32_t b) {
  if constexpr (t < D) {
    prod[t] = at_point8<t>(F, a, b);
    first8<D, t + 1>(F, prod, a, b);
  }
}
template <int D, int t = 0>
__device__ __forceinline__ void factor8(const Tower& F, uint32_t (&prod)[D], uint32_t a, uint32_t b) {
  if constexpr (t < D) {
    prod[t] = F.m8(prod[t], at_point8<t>(F, a, b));
    factor8<D, t + 1>(F, prod, a, b);
  }
}
template <int D, int t = 0>
__device__ __forceinline__ void first128(const Tower& F, g128 (&prod)[D], const g128& a, const g128& b) {
  if constexpr (t < D) {
    prod[t] = at_point128<t>(F, a, b);
    first128<D, t + 1>(F, prod, a, b);
  }
}
template <int D, int t = 0>
__device__ __forceinline__ void factor128(const Tower& F, g128 (&prod)[D], const g128& a, const g128& b) {
  if constexpr (t < D) {
    prod[t] = F.m128(prod[t], at_point128<t>(F, a, b));
    factor128<D, t + 1>(F, prod, a, b);
  }
}

// coefficient * v by the coefficient's kind: v itself, 16 subfield lookups, or a full product
__device__ __forceinline__ g128 times_coef(const Tower& F, uint32_t kind, const g128& c, const g128& v) {
  return kind == 0 ? v : kind == 1 ? F.s128((uint32_t)c.lo, v) : F.m128(c, v);
}

// GF(2^8) round; out: (dmax + 1) bytes packed four to a word (little-endian: byte t is
// values[t]). D > 0: the D = dmax + 1 points in registers, every row once. D = 0: one
// point per pass, points t = blockIdx.y, blockIdx.y + gridDim.y, ... (a grid of dmax + 1
// rows of CTAs gives each point its own CTAs when the rows alone cannot fill the GPU).
template <int D>
__global__ void __launch_bounds__(kBThreads) k_values8(const uint8_t* __restrict__ cur, uint32_t len, uint32_t half,
                                                       uint32_t dmax, const __grid_constant__ Terms tm,
                                                       const uint8_t* __restrict__ gT, uint32_t* __restrict__ out) {
  extern __shared__ uint4 smem_b[];
  uint8_t* s_T = reinterpret_cast<uint8_t*>(smem_b);
  uint32_t* s_acc = reinterpret_cast<uint32_t*>(s_T + 65536);
  const uint32_t words = (dmax + 4) / 4;
  load_table(s_T, gT);
  for (uint32_t k = threadIdx.x; k < words; k += blockDim.x) s_acc[k] = 0;
  __syncthreads();
  const Tower F{s_T};
  const uint32_t stride = gridDim.x * blockDim.x, first = blockIdx.x * blockDim.x + threadIdx.x;
  if constexpr (D > 0) {
    // kRows rows per thread and pass, their loads issued together (the byte loads are
    // latency-bound otherwise); a row past the end loads zeros, whose products are zero
    constexpr int kRows = 4;
    uint32_t acc[D];
#pragma unroll
    for (int t = 0; t < D; ++t) acc[t] = 0;
    for (uint32_t base = first; base < half; base += kRows * stride) {
      uint32_t valid = 0;
#pragma unroll
      for (int r = 0; r < kRows; ++r) valid += base + r * stride < half;
      for (uint32_t k = 0; k < tm.nterms; ++k) {
        const uint32_t j0 = tm.off[k], j1 = tm.off[k + 1], c = tm.coef[k];
        if (j0 == j1) {
#pragma unroll
          for (int t = 0; t < D; ++t) acc[t] ^= (valid & 1) ? c : 0;
          continue;
        }
        uint32_t a[kRows], b[kRows], prod[kRows][D];
        auto load = [&](uint32_t j) {
          const uint8_t* col = cur + (size_t)tm.idx[j] * len;
#pragma unroll
          for (int r = 0; r < kRows; ++r) {
            const uint32_t row = base + r * stride;
            a[r] = row < half ? col[2 * (size_t)row] : 0;
            b[r] = row < half ? col[2 * (size_t)row + 1] : 0;
          }
        };
        load(j0);
#pragma unroll
        for (int r = 0; r < kRows; ++r) {
          first8<D>(F, prod[r], a[r], b[r]);
          if (tm.kind[k] != 0) {
#pragma unroll
            for (int t = 0; t < D; ++t) prod[r][t] = F.m8(c, prod[r][t]);
          }
        }
        for (uint32_t j = j0 + 1; j < j1; ++j) {
          load(j);
#pragma unroll
          for (int r = 0; r < kRows; ++r) factor8<D>(F, prod[r], a[r], b[r]);
        }
#pragma unroll
        for (int r = 0; r < kRows; ++r)
#pragma unroll
          for (int t = 0; t < D; ++t) acc[t] ^= prod[r][t];
      }
    }
#pragma unroll
    for (int t = 0; t < D; ++t) warp_xor_into(acc[t] << (8 * (t & 3)), s_acc + (t >> 2));
  } else {
    for (uint32_t t = blockIdx.y; t <= dmax; t += gridDim.y) {
      uint32_t acc = 0;
      for (uint32_t rest = first; rest < half; rest += stride) {
        for (uint32_t k = 0; k < tm.nterms; ++k) {
          const uint32_t j0 = tm.off[k], j1 = tm.off[k + 1];
          uint32_t prod = tm.coef[k];
          for (uint32_t j = j0; j < j1; ++j) {
            const uint8_t* p = cur + (size_t)tm.idx[j] * len + 2 * (size_t)rest;
            const uint32_t a = p[0], v = a ^ F.m8(t, a ^ p[1]);
            prod = (j == j0 && tm.kind[k] == 0) ? v : F.m8(prod, v);
          }
          acc ^= prod;
        }
      }
      warp_xor_into(acc << (8 * (t & 3)), s_acc + (t >> 2));
    }
  }
  __syncthreads();
  for (uint32_t k = threadIdx.x; k < words; k += blockDim.x)
    if (s_acc[k]) atomicXor(out + k, s_acc[k]);
}

__device__ __forceinline__ g128 load_g128(const uint4* p) {
  const uint4 v = *p;
  return {(uint64_t)v.y << 32 | v.x, (uint64_t)v.w << 32 | v.z};
}

// GF(2^128) round; out: (dmax + 1) values of four little-endian words. D as k_values8.
template <int D>
__global__ void __launch_bounds__(kBThreads, (D >= 1 && D <= 4) ? 2 : 1) k_values128(const uint4* __restrict__ cur, uint32_t len, uint32_t half,
                                                         uint32_t dmax, const __grid_constant__ Terms tm,
                                                         const uint8_t* __restrict__ gT, uint32_t* __restrict__ out) {
  extern __shared__ uint4 smem_b[];
  uint8_t* s_T = reinterpret_cast<uint8_t*>(smem_b);
  uint32_t* s_acc = reinterpret_cast<uint32_t*>(s_T + 65536);
  const uint32_t words = 4 * (dmax + 1);
  load_table(s_T, gT);
  for (uint32_t k = threadIdx.x; k < words; k += blockDim.x) s_acc[k] = 0;
  __syncthreads();
  const Tower F{s_T};
  const uint32_t stride = gridDim.x * blockDim.x, first = blockIdx.x * blockDim.x + threadIdx.x;
  auto coef = [&](uint32_t k) {
    const uint64_t* cf = reinterpret_cast<const uint64_t*>(tm.coef + 16 * k);
    return g128{cf[0], cf[1]};
  };
  if constexpr (D > 0) {
    g128 acc[D];
#pragma unroll
    for (int t = 0; t < D; ++t) acc[t] = {0, 0};
    for (uint32_t rest = first; rest < half; rest += stride) {
      for (uint32_t k = 0; k < tm.nterms; ++k) {
        const uint32_t j0 = tm.off[k], j1 = tm.off[k + 1], kind = tm.kind[k];
        const g128 c = coef(k);
        if (j0 == j1) {
#pragma unroll
          for (int t = 0; t < D; ++t) acc[t] = gxor(acc[t], c);
          continue;
        }
        g128 prod[D];
        const uint4* p = cur + (size_t)tm.idx[j0] * len + 2 * (size_t)rest;
        first128<D>(F, prod, load_g128(p), load_g128(p + 1));
        if (kind != 0) {
#pragma unroll
          for (int t = 0; t < D; ++t) prod[t] = times_coef(F, kind, c, prod[t]);
        }
        for (uint32_t j = j0 + 1; j < j1; ++j) {
          p = cur + (size_t)tm.idx[j] * len + 2 * (size_t)rest;
          factor128<D>(F, prod, load_g128(p), load_g128(p + 1));
        }
#pragma unroll
        for (int t = 0; t < D; ++t) acc[t] = gxor(acc[t], prod[t]);
      }
    }
#pragma unroll
    for (int t = 0; t < D; ++t) warp_xor_into128(acc[t], s_acc + 4 * t);
  } else {
    for (uint32_t t = blockIdx.y; t <= dmax; t += gridDim.y) {
      g128 acc{0, 0};
      for (uint32_t rest = first; rest < half; rest += stride) {
        for (uint32_t k = 0; k < tm.nterms; ++k) {
          const uint32_t j0 = tm.off[k], j1 = tm.off[k + 1], kind = tm.kind[k];
          const g128 c = coef(k);
          g128 prod = c;
          for (uint32_t j = j0; j < j1; ++j) {
            const uint4* p = cur + (size_t)tm.idx[j] * len + 2 * (size_t)rest;
            const g128 a = load_g128(p), v = gxor(a, F.s128(t, gxor(a, load_g128(p + 1))));
            prod = j == j0 ? times_coef(F, kind, c, v) : F.m128(prod, v);
          }
          acc = gxor(acc, prod);
        }
      }
      warp_xor_into128(acc, s_acc + 4 * t);
    }
  }
  __syncthreads();
  for (uint32_t k = threadIdx.x; k < words; k += blockDim.x)
    if (s_acc[k]) atomicXor(out + k, s_acc[k]);
}

// next[f][rest] = a + r (a + b) over GF(2^8); grid.y runs over the tables.
// d_r: the challenge in device memory (the prover's device transcript), else r.
__global__ void __launch_bounds__(kBThreads) k_fold8(const uint8_t* __restrict__ cur, uint32_t len, uint32_t half,
                                                     uint32_t r, const uint8_t* __restrict__ d_r,
                                                     const uint8_t* __restrict__ gT, uint8_t* __restrict__ next) {
  __shared__ uint8_t row[256];
  if (d_r) r = d_r[0];
  for (uint32_t k = threadIdx.x; k < 256; k += blockDim.x) row[k] = gT[(r << 8) | k];
  __syncthreads();
  const uint8_t* src = cur + (size_t)blockIdx.y * len;
  uint8_t* dst = next + (size_t)blockIdx.y * half;
  for (uint32_t rest = blockIdx.x * blockDim.x + threadIdx.x; rest < half; rest += gridDim.x * blockDim.x) {
    const uint32_t a = src[2 * (size_t)rest], b = src[2 * (size_t)rest + 1];
    dst[rest] = (uint8_t)(a ^ row[a ^ b]);
  }
}

// R[k][v] = r * (v at byte k), the GF(2^8)-linear map x -> r x on byte coordinates.
__global__ void __launch_bounds__(kBThreads) k_mul_table128(uint64_t r_lo, uint64_t r_hi, const uint8_t* __restrict__ d_r,
                                                            const uint8_t* __restrict__ gT, uint4* __restrict__ R) {
  extern __shared__ uint4 smem_b[];
  if (d_r) {  // the challenge in device memory: 16 little-endian bytes
    r_lo = r_hi = 0;
    for (int b = 7; b >= 0; --b) r_lo = (r_lo << 8) | d_r[b], r_hi = (r_hi << 8) | d_r[8 + b];
  }
  uint8_t* s_T = reinterpret_cast<uint8_t*>(smem_b);
  load_table(s_T, gT);
  __syncthreads();
  const Tower F{s_T};
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;  // < 4096 by the launch
  const uint32_t k = i >> 8, v = i & 255;
  const g128 x{k < 8 ? (uint64_t)v << (8 * k) : 0, k >= 8 ? (uint64_t)v << (8 * (k - 8)) : 0};
  const g128 p = F.m128(g128{r_lo, r_hi}, x);
  R[i] = make_uint4((uint32_t)p.lo, (uint32_t)(p.lo >> 32), (uint32_t)p.hi, (uint32_t)(p.hi >> 32));
}

__global__ void __launch_bounds__(kBThreads) k_fold128(const uint4* __restrict__ cur, uint32_t len, uint32_t half,
                                                       const uint4* __restrict__ R, uint4* __restrict__ next) {
  extern __shared__ uint4 smem_b[];
  uint4* s_R = smem_b;
  for (uint32_t k = threadIdx.x; k < 4096; k += blockDim.x) s_R[k] = R[k];
  __syncthreads();
  const uint4* src = cur + (size_t)blockIdx.y * len;
  uint4* dst = next + (size_t)blockIdx.y * half;
  for (uint32_t rest = blockIdx.x * blockDim.x + threadIdx.x; rest < half; rest += gridDim.x * blockDim.x) {
    const uint4 a = src[2 * (size_t)rest], b = src[2 * (size_t)rest + 1];
    const uint32_t d[4] = {a.x ^ b.x, a.y ^ b.y, a.z ^ b.z, a.w ^ b.w};
    uint4 o = a;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const uint4 e = s_R[(k << 8) | ((d[k >> 2] >> (8 * (k & 3))) & 0xff)];
      o.x ^= e.x, o.y ^= e.y, o.z ^= e.z, o.w ^= e.w;
    }
    dst[rest] = o;
  }
}

// ---- device: one round's transcript step of the combination prover ----------------
// After a round's values are on the device: the round's coefficients by the Lagrange
// matrix (sumcheck.zig:124-162), then the SHA-256 transcript step (sumcheck.zig:66-87)
// that absorbs them and samples the next challenge, so the rounds of a proof run back to
// back on the device with no trip to the host between them.

__constant__ uint32_t kSha256K[64] = {
    0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5,
    0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174,
    0xe49b69c1, 0xefbe4786, 0x0fc19dc6, 0x240ca1cc, 0x2de92c6f, 0x4a7484aa, 0x5cb0a9dc, 0x76f988da,
    0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7, 0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967,
    0x27b70a85, 0x2e1b2138, 0x4d2c6dfc, 0x53380d13, 0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85,
    0xa2bfe8a1, 0xa81a664b, 0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070,
    0x19a4c116, 0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a, 0x5b9cca4f, 0x682e6ff3,
    0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7, 0xc67178f2};

// SHA-256 (FIPS 180-4) of the message prefix || body in one thread. Each 64-byte block's
// words are assembled from the message bytes (and the padding, computed on the fly), and
// the 64 rounds are unrolled so the message schedule stays in registers.
__device__ __forceinline__ uint32_t sha_rotr(uint32_t x, unsigned r) { return __funnelshift_r(x, x, r); }

__device__ void sha256_dev(const uint8_t* prefix, uint32_t plen, const uint8_t* body, uint32_t blen,
                           uint8_t out[32]) {
  uint32_t h[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a, 0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};
  const uint64_t len = (uint64_t)plen + blen;
  const uint64_t nblocks = (len + 9 + 63) / 64;
  const uint64_t bits = len * 8;
  auto byte_at = [&](uint64_t i) -> uint32_t {
    if (i < plen) return prefix[i];
    if (i < len) return body[i - plen];
    if (i == len) return 0x80;
    const uint64_t end = nblocks * 64;
    if (i >= end - 8) return (uint32_t)(bits >> (8 * (end - 1 - i))) & 0xff;
    return 0;
  };
  for (uint64_t blk = 0; blk < nblocks; ++blk) {
    uint32_t w[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const uint64_t o = blk * 64 + 4 * i;
      w[i] = byte_at(o) << 24 | byte_at(o + 1) << 16 | byte_at(o + 2) << 8 | byte_at(o + 3);
    }
    uint32_t a = h[0], b = h[1], c = h[2], d = h[3], e = h[4], f = h[5], g = h[6], hh = h[7];
#pragma unroll
    for (int i = 0; i < 64; ++i) {
      if (i >= 16) {
        const uint32_t x = w[(i - 15) & 15], y = w[(i - 2) & 15];
        w[i & 15] += (sha_rotr(x, 7) ^ sha_rotr(x, 18) ^ (x >> 3)) + w[(i - 7) & 15] +
                     (sha_rotr(y, 17) ^ sha_rotr(y, 19) ^ (y >> 10));
      }
      const uint32_t t1 =
          hh + (sha_rotr(e, 6) ^ sha_rotr(e, 11) ^ sha_rotr(e, 25)) + ((e & f) ^ (~e & g)) + kSha256K[i] + w[i & 15];
      const uint32_t t2 = (sha_rotr(a, 2) ^ sha_rotr(a, 13) ^ sha_rotr(a, 22)) + ((a & b) ^ (a & c) ^ (b & c));
      hh = g, g = f, f = e, e = d + t1, d = c, c = b, b = a, a = t1 + t2;
    }
    h[0] += a, h[1] += b, h[2] += c, h[3] += d, h[4] += e, h[5] += f, h[6] += g, h[7] += hh;
  }
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) out[4 * i + j] = (uint8_t)(h[i] >> (24 - 8 * j));
}

// The device transcript: the SHA-256 state (32 bytes) and the last challenge (1 or 16
// bytes), in device memory between rounds.
struct ScTranscript {
  uint8_t state[32];
  uint8_t r[16];
};

// Round `round`'s step. The points 0..n-1 lie in GF(2^8), so the Lagrange matrix `lag`
// (n x n bytes) does too, and coefficient d = sum_i values[i] * lag[i][d] takes products by
// a subfield scalar (one lookup over GF(2^8), 16 independent ones over GF(2^128)); one lane
// per coefficient, the product table in global memory. The coefficients go to rounds_out;
// the first round also forms the claimed sum (values[0] + values[1]) and starts the
// transcript (from `seed`, or from the claimed sum); then thread 0 absorbs the
// coefficients and samples the challenge (the digest's last byte over GF(2^8), its last
// 16 bytes over GF(2^128)).
template <bool WIDE>
__global__ void __launch_bounds__(64) k_sc_step(const uint8_t* __restrict__ vals, const uint8_t* __restrict__ lag,
                                                uint32_t n, uint32_t round, const uint8_t* __restrict__ gT,
                                                const uint8_t* __restrict__ seed, uint32_t seed_len, int has_seed,
                                                ScTranscript* __restrict__ tx, uint8_t* __restrict__ claimed,
                                                uint8_t* __restrict__ rounds_out) {
  constexpr uint32_t ES = WIDE ? 16 : 1;
  __shared__ uint8_t s_msg[32 + kProveMaxPoints * 16];  // the absorbed message: state || coefficients
  const Tower F{gT};
  for (uint32_t d = threadIdx.x; d < n; d += blockDim.x) {
    uint8_t* out = s_msg + 32 + ES * d;
    if constexpr (WIDE) {
      uint64_t lo = 0, hi = 0;
      for (uint32_t i = 0; i < n; ++i) {
        const uint32_t c = lag[(size_t)i * n + d];
        const uint8_t* v = vals + 16 * i;
        uint64_t vlo = 0, vhi = 0;
#pragma unroll
        for (int b = 7; b >= 0; --b) vlo = (vlo << 8) | v[b], vhi = (vhi << 8) | v[8 + b];
        lo ^= F.s64(c, vlo);
        hi ^= F.s64(c, vhi);
      }
#pragma unroll
      for (int b = 0; b < 8; ++b) out[b] = (uint8_t)(lo >> (8 * b)), out[8 + b] = (uint8_t)(hi >> (8 * b));
    } else {
      uint32_t acc = 0;
      for (uint32_t i = 0; i < n; ++i) acc ^= F.m8(lag[(size_t)i * n + d], vals[i]);
      out[0] = (uint8_t)acc;
    }
    for (uint32_t b = 0; b < ES; ++b) rounds_out[((size_t)round * n + d) * ES + b] = out[b];
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  if (round == 0) {
    uint8_t h[16];
    for (uint32_t b = 0; b < ES; ++b) {  // one point: the sum of 2^k copies of a constant is 0
      h[b] = n >= 2 ? (uint8_t)(vals[b] ^ vals[ES + b]) : 0;
      claimed[b] = h[b];
    }
    if (has_seed)
      sha256_dev(seed, seed_len, nullptr, 0, s_msg);
    else
      sha256_dev(h, ES, nullptr, 0, s_msg);
  } else {
    for (int b = 0; b < 32; ++b) s_msg[b] = tx->state[b];
  }
  uint8_t st[32];
  sha256_dev(s_msg, 32 + n * ES, nullptr, 0, st);
  for (int b = 0; b < 32; ++b) tx->state[b] = st[b];
  for (uint32_t b = 0; b < ES; ++b) tx->r[b] = WIDE ? st[16 + b] : st[31];
}

// ---- host: argument checks and launches -------------------------------------------

Terms pack_terms(bool wide, size_t m, const uint8_t* coeffs, size_t nterms, const uint32_t* indices,
                 size_t n_indices, const uint32_t* offsets) {
  if (!coeffs || !offsets || (n_indices && !indices)) throw Error(ZS_EMALFORMED, "null terms");
  if (nterms == 0 || nterms > kMaxTerms || n_indices > kMaxFactors) throw Error(ZS_EMALFORMED, "too many terms");
  if (m == 0 || m > kMaxTables) throw Error(ZS_EMALFORMED, "table count");
  if (offsets[0] != 0 || offsets[nterms] != n_indices) throw Error(ZS_EMALFORMED, "term offsets");
  Terms tm;
  std::memset(&tm, 0, sizeof(tm));
  tm.nterms = (uint32_t)nterms;
  for (size_t k = 0; k <= nterms; ++k) {
    if (k && offsets[k] < offsets[k - 1]) throw Error(ZS_EMALFORMED, "term offsets");
    tm.off[k] = offsets[k];
  }
  for (size_t j = 0; j < n_indices; ++j) {
    if (indices[j] >= m) throw Error(ZS_EMALFORMED, "factor table out of range");
    tm.idx[j] = (uint16_t)indices[j];
  }
  const size_t es = wide ? 16 : 1;
  std::memcpy(tm.coef, coeffs, nterms * es);
  for (size_t k = 0; k < nterms; ++k) {
    bool high_zero = true;  // the coefficient lies in GF(2^8)
    for (size_t b = 1; b < es; ++b) high_zero = high_zero && coeffs[es * k + b] == 0;
    tm.kind[k] = high_zero && coeffs[es * k] == 1 ? 0 : (wide && high_zero ? 1 : 2);
  }
  return tm;
}

void check_rows(size_t len, size_t half, size_t dmax) {
  if (2 * half > len || len > 0xffffffffu) throw Error(ZS_EMALFORMED, "table length");
  if (dmax > kMaxPoint) throw Error(ZS_EMALFORMED, "more than 256 points");
}

// The values kernels by point count (index D, 0 = one point per pass) and the shared
// memory they are launched with at most: the table and the largest accumulator.
const void* const kValues8[kRegPoints + 1] = {
    (const void*)k_values8<0>, (const void*)k_values8<1>, (const void*)k_values8<2>,
    (const void*)k_values8<3>, (const void*)k_values8<4>, (const void*)k_values8<5>,
    (const void*)k_values8<6>, (const void*)k_values8<7>, (const void*)k_values8<8>};
const void* const kValues128[kRegPoints + 1] = {
    (const void*)k_values128<0>, (const void*)k_values128<1>, (const void*)k_values128<2>,
    (const void*)k_values128<3>, (const void*)k_values128<4>, (const void*)k_values128<5>,
    (const void*)k_values128<6>, (const void*)k_values128<7>, (const void*)k_values128<8>};
constexpr size_t kValuesSmem = 65536 + 16 * (kMaxPoint + 1);

// Per device, set up on first use: the product table, the SM count, the kernels' shared
// memory limits and how many CTAs of each fit on an SM.
struct DeviceState {
  uint8_t* table = nullptr;
  int sms = 0;
  int per_sm8[kRegPoints + 1] = {}, per_sm128[kRegPoints + 1] = {};
};
std::mutex g_dev_mu;
DeviceState g_dev[64];

const DeviceState& device_state(cudaStream_t st) {
  int dev = 0;
  ZS_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) throw Error(ZS_EDEVICE, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_dev_mu);
  DeviceState& d = g_dev[dev];
  if (!d.table) {
    ZS_CUDA(cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev));
    for (int D = 0; D <= kRegPoints; ++D) {
      for (int w = 0; w < 2; ++w) {
        const void* fn = w ? kValues128[D] : kValues8[D];
        int* per_sm = w ? &d.per_sm128[D] : &d.per_sm8[D];
        ZS_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kValuesSmem));
        ZS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, fn, kBThreads, kValuesSmem));
        *per_sm = std::max(*per_sm, 1);
      }
    }
    ZS_CUDA(cudaFuncSetAttribute(k_mul_table128, cudaFuncAttributeMaxDynamicSharedMemorySize, 65536));
    ZS_CUDA(cudaFuncSetAttribute(k_fold128, cudaFuncAttributeMaxDynamicSharedMemorySize, 65536));
    uint8_t* t = nullptr;
    ZS_CUDA(cudaMalloc(&t, 65536));
    ZS_CUDA(cudaMemcpyAsync(t, host_tower().T.data(), 65536, cudaMemcpyHostToDevice, st));
    ZS_CUDA(cudaStreamSynchronize(st));
    d.table = t;
  }
  return d;
}

// Zeroes d_out and accumulates one round's values into it, asynchronously on `st`. With
// enough rows to give every SM a CTA, each thread takes all points of its rows (up to
// eight; one point per pass beyond that); with fewer rows, the points get CTAs of their
// own (a grid of dmax + 1 rows), so that small rounds still spread over the GPU.
void values_async(bool wide, const void* d_cur, size_t len, size_t half, size_t dmax, const Terms& tm, void* d_out,
                  cudaStream_t st) {
  const size_t words = wide ? 4 * (dmax + 1) : (dmax + 4) / 4;
  ZS_CUDA(cudaMemsetAsync(d_out, 0, words * 4, st));
  if (half == 0) return;
  const DeviceState& ds = device_state(st);
  const int D = dmax + 1 <= (size_t)kRegPoints ? (int)dmax + 1 : 0;
  const size_t row_blocks = (half + kBThreads - 1) / kBThreads;
  const bool per_row = D > 0 && row_blocks >= (size_t)ds.sms;
  const int kd = per_row ? D : 0;
  const size_t slots = (size_t)ds.sms * (wide ? ds.per_sm128[kd] : ds.per_sm8[kd]);
  dim3 grid(1, 1);
  if (per_row) {
    grid.x = (unsigned)std::min(row_blocks, slots);
  } else {
    grid.y = (unsigned)(dmax + 1);
    grid.x = (unsigned)std::min(row_blocks, std::max<size_t>(1, (slots + dmax) / (dmax + 1)));
  }
  const void* cur = d_cur;
  uint32_t L = (uint32_t)len, H = (uint32_t)half, M = (uint32_t)dmax;
  const uint8_t* T = ds.table;
  uint32_t* out = static_cast<uint32_t*>(d_out);
  void* args[] = {&cur, &L, &H, &M, const_cast<Terms*>(&tm), &T, &out};
  ZS_CUDA(cudaLaunchKernel(wide ? kValues128[kd] : kValues8[kd], grid, dim3(kBThreads), args, 65536 + 4 * words,
                           st));
}

// next (m tables of len / 2) = fold of cur (m tables of len) at r, asynchronously on `st`.
// r_mul: a 64 KB device buffer for the GF(2^128) multiply table.
void fold_async(bool wide, const void* d_cur, size_t len, size_t m, u128 r, const uint8_t* d_r, void* d_next,
                uint4* r_mul, cudaStream_t st) {
  const size_t half = len / 2;
  if (half == 0) return;
  const DeviceState& ds = device_state(st);
  const uint32_t bx = (uint32_t)std::min<size_t>((half + kBThreads - 1) / kBThreads,
                                                 std::max<size_t>(1, (size_t)ds.sms * 8 / m));
  const dim3 grid(bx, (unsigned)m);
  if (!wide) {
    k_fold8<<<grid, kBThreads, 0, st>>>(static_cast<const uint8_t*>(d_cur), (uint32_t)len, (uint32_t)half,
                                        (uint32_t)r, d_r, ds.table, static_cast<uint8_t*>(d_next));
  } else {
    k_mul_table128<<<4096 / kBThreads, kBThreads, 65536, st>>>((uint64_t)r, (uint64_t)(r >> 64), d_r, ds.table, r_mul);
    k_fold128<<<grid, kBThreads, 65536, st>>>(static_cast<const uint4*>(d_cur), (uint32_t)len, (uint32_t)half,
                                              r_mul, static_cast<uint4*>(d_next));
  }
  ZS_CUDA(cudaGetLastError());
}

template <typename T>
struct DevMem {
  T* p = nullptr;
  cudaStream_t st;
  DevMem(size_t n, cudaStream_t s) : st(s) { ZS_CUDA(cudaMallocAsync((void**)&p, n ? n * sizeof(T) : 1, s)); }
  ~DevMem() {
    if (p) cudaFreeAsync(p, st);
  }
  DevMem(const DevMem&) = delete;
  DevMem& operator=(const DevMem&) = delete;
};

template <typename F>
int32_t guarded(F&& f) {
  try {
    f();
    return ZS_OK;
  } catch (const Error& e) {
    return e.code;
  } catch (const std::bad_alloc&) {
    return ZS_ENOMEM;
  } catch (...) {
    return ZS_EGENERIC;
  }
}

bool field_wide(uint32_t field_bits) {
  if (field_bits != 8 && field_bits != 128) throw Error(ZS_EMALFORMED, "field_bits is 8 or 128");
  return field_bits == 128;
}

int32_t hook_values(bool wide, const uint8_t* cur_flat, size_t len, size_t m, const uint8_t* coeffs, size_t nterms,
                    const uint32_t* indices, size_t n_indices, const uint32_t* offsets, size_t dmax, size_t half,
                    uint8_t* out, void* stream) {
  return guarded([&] {
    if (!cur_flat || !out) throw Error(ZS_EMALFORMED, "null buffer");
    check_rows(len, half, dmax);
    const Terms tm = pack_terms(wide, m, coeffs, nterms, indices, n_indices, offsets);
    cudaStream_t st = (cudaStream_t)stream;
    const size_t es = wide ? 16 : 1, words = wide ? 4 * (dmax + 1) : (dmax + 4) / 4;
    DevMem<uint4> d_cur((m * len * es + 15) / 16, st);
    DevMem<uint32_t> d_out(words, st);
    if (m * len) ZS_CUDA(cudaMemcpyAsync(d_cur.p, cur_flat, m * len * es, cudaMemcpyHostToDevice, st));
    values_async(wide, d_cur.p, len, half, dmax, tm, d_out.p, st);
    std::vector<uint32_t> h(words);
    ZS_CUDA(cudaMemcpyAsync(h.data(), d_out.p, words * 4, cudaMemcpyDeviceToHost, st));
    ZS_CUDA(cudaStreamSynchronize(st));
    std::memcpy(out, h.data(), (dmax + 1) * es);
  });
}

// ---- host: the combination prover (sumcheck.zig:208-395) ---------------------------

u128 load_elem(const uint8_t* p, size_t es) {
  u128 v = 0;
  for (size_t i = es; i-- > 0;) v = (v << 8) | p[i];
  return v;
}
void store_elem(uint8_t* p, size_t es, u128 v) {
  for (size_t i = 0; i < es; ++i) p[i] = (uint8_t)(v >> (8 * i));
}

// Lagrange interpolation through the points 0..n-1 (sumcheck.zig:124-162) as a matrix:
// row i holds the low-first coefficients of prod_{j != i} (x + j) / (i + j), so a round's
// coefficients are coeffs[d] = sum_i values[i] * lag[i][d] (k_sc_step). The matrix
// depends on the points only and is built once per proof, on the host.
std::vector<std::vector<u128>> lagrange_matrix(const HostTower& ht, unsigned level, size_t n) {
  std::vector<std::vector<u128>> lag(n, std::vector<u128>(n, 0));
  for (size_t i = 0; i < n; ++i) {
    std::vector<u128> basis{1};
    u128 denom = 1;
    for (size_t j = 0; j < n; ++j) {
      if (j == i) continue;
      std::vector<u128> next(basis.size() + 1, 0);  // basis * (x + j)
      for (size_t d = 0; d < basis.size(); ++d) {
        next[d + 1] ^= basis[d];
        next[d] ^= ht.mul(level, (u128)j, basis[d]);
      }
      basis.swap(next);
      denom = ht.mul(level, denom, (u128)(i ^ j));
    }
    const u128 inv = ht.inv(level, denom);
    for (size_t d = 0; d < n; ++d) lag[i][d] = ht.mul(level, basis[d], inv);
  }
  return lag;
}

int32_t prove_combination(uint32_t field_bits, const uint8_t* tables, size_t k, size_t m, const uint8_t* coeffs,
                          size_t nterms, const uint32_t* indices, size_t n_indices, const uint32_t* offsets,
                          const uint8_t* seed, size_t seed_len, int32_t has_seed, uint8_t* claimed_out,
                          uint8_t* rounds_out, void* stream) {
  return guarded([&] {
    const bool wide = field_wide(field_bits);
    const unsigned level = wide ? 7 : 3;
    const size_t es = wide ? 16 : 1;
    if (!tables || !claimed_out || (k && !rounds_out) || (has_seed && seed_len && !seed))
      throw Error(ZS_EMALFORMED, "null buffer");
    if (k > 31) throw Error(ZS_EMALFORMED, "more than 2^31 rows");
    const Terms tm = pack_terms(wide, m, coeffs, nterms, indices, n_indices, offsets);
    size_t dmax = 0;
    for (size_t t = 0; t < nterms; ++t) dmax = std::max<size_t>(dmax, offsets[t + 1] - offsets[t]);
    if (dmax + 1 > kProveMaxPoints) throw Error(ZS_EMALFORMED, "more than 64 points");
    const size_t n = (size_t)1 << k;
    if (m > (((size_t)1 << 36) / es) / n) throw Error(ZS_EMALFORMED, "tables larger than 64 GB");
    const HostTower& ht = host_tower();

    if (k == 0) {  // one row: the claimed sum is g at it, no rounds
      u128 h = 0;
      for (size_t t = 0; t < nterms; ++t) {
        u128 p = load_elem(coeffs + es * t, es);
        for (uint32_t j = offsets[t]; j < offsets[t + 1]; ++j) p = ht.mul(level, p, load_elem(tables + es * indices[j], es));
        h ^= p;
      }
      store_elem(claimed_out, es, h);
      return;
    }

    const std::vector<std::vector<u128>> lag = lagrange_matrix(ht, 3, dmax + 1);  // in GF(2^8) (points < 256)

    cudaStream_t st = (cudaStream_t)stream;
    retain_pool_memory();
    const size_t words = wide ? 4 * (dmax + 1) : (dmax + 4) / 4;
    DevMem<uint4> d_a((m * n * es + 15) / 16, st), d_b((m * (n / 2) * es + 15) / 16, st);
    DevMem<uint32_t> d_vals(words, st);
    DevMem<uint4> d_rmul(wide ? 4096 : 0, st);
    // the device transcript's inputs and outputs: the Lagrange matrix, the seed, the
    // state and challenge, the claimed sum and every round's coefficients
    const size_t pts = dmax + 1;
    std::vector<uint8_t> lag_b(pts * pts);  // GF(2^8) entries: the points lie in GF(2^8)
    for (size_t a = 0; a < pts; ++a)
      for (size_t d = 0; d < pts; ++d) lag_b[a * pts + d] = (uint8_t)lag[a][d];
    DevMem<uint8_t> d_lag(lag_b.size(), st), d_seed(has_seed ? seed_len : 0, st), d_claimed(es, st),
        d_rounds(k * pts * es, st);
    DevMem<ScTranscript> d_tx(1, st);
    ZS_CUDA(cudaMemcpyAsync(d_lag.p, lag_b.data(), lag_b.size(), cudaMemcpyHostToDevice, st));
    if (has_seed && seed_len) ZS_CUDA(cudaMemcpyAsync(d_seed.p, seed, seed_len, cudaMemcpyHostToDevice, st));
    ZS_CUDA(cudaMemcpyAsync(d_a.p, tables, m * n * es, cudaMemcpyHostToDevice, st));
    const uint8_t* T = device_state(st).table;

    // every round on the device, back to back: values, the transcript step, the fold
    void* cur = d_a.p;
    void* nxt = d_b.p;
    size_t len = n;
    for (size_t i = 0; i < k; ++i) {
      const size_t half = len / 2;
      values_async(wide, cur, len, half, dmax, tm, d_vals.p, st);
      const uint8_t* vb = reinterpret_cast<const uint8_t*>(d_vals.p);
      if (wide)
        k_sc_step<true><<<1, 64, 0, st>>>(vb, d_lag.p, (uint32_t)pts, (uint32_t)i, T, d_seed.p, (uint32_t)seed_len,
                                          has_seed ? 1 : 0, d_tx.p, d_claimed.p, d_rounds.p);
      else
        k_sc_step<false><<<1, 64, 0, st>>>(vb, d_lag.p, (uint32_t)pts, (uint32_t)i, T, d_seed.p, (uint32_t)seed_len,
                                           has_seed ? 1 : 0, d_tx.p, d_claimed.p, d_rounds.p);
      ZS_CUDA(cudaGetLastError());
      if (i + 1 < k) {
        fold_async(wide, cur, len, m, 0, reinterpret_cast<const uint8_t*>(d_tx.p) + offsetof(ScTranscript, r), nxt,
                   d_rmul.p, st);
        std::swap(cur, nxt);
      }
      len = half;
    }
    ZS_CUDA(cudaMemcpyAsync(claimed_out, d_claimed.p, es, cudaMemcpyDeviceToHost, st));
    ZS_CUDA(cudaMemcpyAsync(rounds_out, d_rounds.p, k * pts * es, cudaMemcpyDeviceToHost, st));
    ZS_CUDA(cudaStreamSynchronize(st));
  });
}

}  // namespace
}  // namespace zs

extern "C" int32_t zs_binius_sumcheck_values_gf256(const uint8_t* cur_flat, size_t len, size_t m,
                                                   const uint8_t* coeffs, size_t nterms, const uint32_t* indices,
                                                   size_t n_indices, const uint32_t* offsets, size_t dmax, size_t half,
                                                   uint8_t* out, void* stream) {
  return zs::hook_values(false, cur_flat, len, m, coeffs, nterms, indices, n_indices, offsets, dmax, half, out,
                         stream);
}

extern "C" int32_t zs_binius_sumcheck_values_gf128(const uint8_t* cur_flat, size_t len, size_t m,
                                                   const uint8_t* coeffs, size_t nterms, const uint32_t* indices,
                                                   size_t n_indices, const uint32_t* offsets, size_t dmax,
                                                   size_t half, uint8_t* out, void* stream) {
  return zs::hook_values(true, cur_flat, len, m, coeffs, nterms, indices, n_indices, offsets, dmax, half, out,
                         stream);
}

extern "C" int32_t zs_binius_sumcheck_values_device(uint32_t field_bits, const void* d_cur, size_t len, size_t m,
                                                    const uint8_t* coeffs, size_t nterms, const uint32_t* indices,
                                                    size_t n_indices, const uint32_t* offsets, size_t dmax,
                                                    size_t half, void* d_out, void* stream) {
  return zs::guarded([&] {
    const bool wide = zs::field_wide(field_bits);
    if (!d_cur || !d_out) throw zs::Error(zs::ZS_EMALFORMED, "null buffer");
    if ((reinterpret_cast<uintptr_t>(d_out) & 3) || (wide && (reinterpret_cast<uintptr_t>(d_cur) & 15)))
      throw zs::Error(zs::ZS_EMALFORMED, "misaligned buffer");
    zs::check_rows(len, half, dmax);
    const zs::Terms tm = zs::pack_terms(wide, m, coeffs, nterms, indices, n_indices, offsets);
    zs::values_async(wide, d_cur, len, half, dmax, tm, d_out, (cudaStream_t)stream);
  });
}

extern "C" int32_t zs_binius_sumcheck_fold_device(uint32_t field_bits, const void* d_cur, size_t len, size_t m,
                                                  const uint8_t* r, void* d_next, void* d_scratch, void* stream) {
  return zs::guarded([&] {
    const bool wide = zs::field_wide(field_bits);
    if (!d_cur || !d_next || !r || (wide && !d_scratch)) throw zs::Error(zs::ZS_EMALFORMED, "null buffer");
    if (wide && ((reinterpret_cast<uintptr_t>(d_cur) | reinterpret_cast<uintptr_t>(d_next) |
                  reinterpret_cast<uintptr_t>(d_scratch)) & 15))
      throw zs::Error(zs::ZS_EMALFORMED, "misaligned buffer");
    if (len > 0xffffffffu || m == 0 || m > zs::kMaxTables) throw zs::Error(zs::ZS_EMALFORMED, "table shape");
    zs::fold_async(wide, d_cur, len, m, zs::load_elem(r, wide ? 16 : 1), nullptr, d_next,
                   static_cast<uint4*>(d_scratch),
                   (cudaStream_t)stream);
  });
}

extern "C" int32_t zs_binius_sumcheck_prove_combination(uint32_t field_bits, const uint8_t* tables, size_t k,
                                                        size_t m, const uint8_t* coeffs, size_t nterms,
                                                        const uint32_t* indices, size_t n_indices,
                                                        const uint32_t* offsets, const uint8_t* seed,
                                                        size_t seed_len, int32_t has_seed, uint8_t* claimed_out,
                                                        uint8_t* rounds_out, void* stream) {
  return zs::prove_combination(field_bits, tables, k, m, coeffs, nterms, indices, n_indices, offsets, seed,
                               seed_len, has_seed, claimed_out, rounds_out, stream);
}
