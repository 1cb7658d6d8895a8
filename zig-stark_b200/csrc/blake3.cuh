// BLAKE3 compression (unkeyed hash mode, 32-byte output) for host and device.
//
// The reference hashes with Zig's std.crypto.hash.Blake3 (src/core/hash/hash.zig:9-24,
// src/m31/hash.zig:16-24, src/core/channel/channel.zig:12-21). On the device every
// compression runs in one thread on the integer pipes: the 16-word state and message
// stay in registers, the 7 rounds are unrolled with the per-round message schedule
// resolved at compile time, and the 16/8-bit rotations are byte permutes.
//
// Messages on this path are short (16-byte QM31 leaves, 78-byte Merkle nodes,
// 4*cols-byte row leaves), so the device helpers below cover single-chunk inputs
// (<= 1024 bytes) only. The host-side incremental hasher (`Hasher`) handles any length
// and is what the Fiat-Shamir transcript uses.
#pragma once
#include <cstdint>
#include <cstring>

#include "field.cuh"

namespace zs {
namespace b3 {

constexpr uint32_t IV0 = 0x6A09E667u, IV1 = 0xBB67AE85u, IV2 = 0x3C6EF372u, IV3 = 0xA54FF53Au,
                   IV4 = 0x510E527Fu, IV5 = 0x9B05688Cu, IV6 = 0x1F83D9ABu, IV7 = 0x5BE0CD19u;
constexpr uint32_t CHUNK_START = 1, CHUNK_END = 2, PARENT = 4, ROOT = 8;

ZS_HD uint32_t rotr16(uint32_t x) {
#ifdef __CUDA_ARCH__
  return __byte_perm(x, 0, 0x1032);
#else
  return (x >> 16) | (x << 16);
#endif
}
ZS_HD uint32_t rotr8(uint32_t x) {
#ifdef __CUDA_ARCH__
  return __byte_perm(x, 0, 0x0321);
#else
  return (x >> 8) | (x << 24);
#endif
}
ZS_HD uint32_t rotr12(uint32_t x) {
#ifdef __CUDA_ARCH__
  return __funnelshift_r(x, x, 12);
#else
  return (x >> 12) | (x << 20);
#endif
}
ZS_HD uint32_t rotr7(uint32_t x) {
#ifdef __CUDA_ARCH__
  return __funnelshift_r(x, x, 7);
#else
  return (x >> 7) | (x << 25);
#endif
}

#define ZS_B3_G(a, b, c, d, mx, my) \
  a = a + b + (mx);                 \
  d = rotr16(d ^ a);                \
  c = c + d;                        \
  b = rotr12(b ^ c);                \
  a = a + b + (my);                 \
  d = rotr8(d ^ a);                 \
  c = c + d;                        \
  b = rotr7(b ^ c);

// Message word order of each round (round r uses the permutation applied r times).
#define ZS_B3_ROUND(m, s0, s1, s2, s3, s4, s5, s6, s7, s8, s9, s10, s11, s12, s13, s14, s15) \
  ZS_B3_G(v0, v4, v8, v12, m[s0], m[s1])                                                   \
  ZS_B3_G(v1, v5, v9, v13, m[s2], m[s3])                                                   \
  ZS_B3_G(v2, v6, v10, v14, m[s4], m[s5])                                                  \
  ZS_B3_G(v3, v7, v11, v15, m[s6], m[s7])                                                  \
  ZS_B3_G(v0, v5, v10, v15, m[s8], m[s9])                                                  \
  ZS_B3_G(v1, v6, v11, v12, m[s10], m[s11])                                                \
  ZS_B3_G(v2, v7, v8, v13, m[s12], m[s13])                                                 \
  ZS_B3_G(v3, v4, v9, v14, m[s14], m[s15])

// Compression returning the 8-word chaining value (the first half of the output
// state): cv <- compress(cv, m, counter = 0, block_len, flags)[0..8]. Every call on
// this path uses counter 0 (single-chunk messages and parent nodes).
ZS_HD void compress_cv(uint32_t cv[8], const uint32_t m[16], uint32_t block_len, uint32_t flags) {
  uint32_t v0 = cv[0], v1 = cv[1], v2 = cv[2], v3 = cv[3], v4 = cv[4], v5 = cv[5], v6 = cv[6], v7 = cv[7];
  uint32_t v8 = IV0, v9 = IV1, v10 = IV2, v11 = IV3, v12 = 0, v13 = 0, v14 = block_len, v15 = flags;
  ZS_B3_ROUND(m, 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15)
  ZS_B3_ROUND(m, 2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8)
  ZS_B3_ROUND(m, 3, 4, 10, 12, 13, 2, 7, 14, 6, 5, 9, 0, 11, 15, 8, 1)
  ZS_B3_ROUND(m, 10, 7, 12, 9, 14, 3, 13, 15, 4, 0, 11, 2, 5, 8, 1, 6)
  ZS_B3_ROUND(m, 12, 13, 9, 11, 15, 10, 14, 8, 7, 2, 5, 3, 0, 1, 6, 4)
  ZS_B3_ROUND(m, 9, 14, 11, 5, 8, 12, 15, 1, 13, 3, 0, 10, 2, 6, 4, 7)
  ZS_B3_ROUND(m, 11, 15, 5, 0, 1, 9, 8, 6, 14, 10, 2, 12, 3, 4, 7, 13)
  cv[0] = v0 ^ v8;
  cv[1] = v1 ^ v9;
  cv[2] = v2 ^ v10;
  cv[3] = v3 ^ v11;
  cv[4] = v4 ^ v12;
  cv[5] = v5 ^ v13;
  cv[6] = v6 ^ v14;
  cv[7] = v7 ^ v15;
}

// Full compression with a 64-bit counter and the 16-word output (host transcript).
ZS_HD void compress_full(const uint32_t cv[8], const uint32_t m[16], uint64_t counter,
                         uint32_t block_len, uint32_t flags, uint32_t out[16]) {
  uint32_t v0 = cv[0], v1 = cv[1], v2 = cv[2], v3 = cv[3], v4 = cv[4], v5 = cv[5], v6 = cv[6], v7 = cv[7];
  uint32_t v8 = IV0, v9 = IV1, v10 = IV2, v11 = IV3;
  uint32_t v12 = (uint32_t)counter, v13 = (uint32_t)(counter >> 32), v14 = block_len, v15 = flags;
  ZS_B3_ROUND(m, 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15)
  ZS_B3_ROUND(m, 2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8)
  ZS_B3_ROUND(m, 3, 4, 10, 12, 13, 2, 7, 14, 6, 5, 9, 0, 11, 15, 8, 1)
  ZS_B3_ROUND(m, 10, 7, 12, 9, 14, 3, 13, 15, 4, 0, 11, 2, 5, 8, 1, 6)
  ZS_B3_ROUND(m, 12, 13, 9, 11, 15, 10, 14, 8, 7, 2, 5, 3, 0, 1, 6, 4)
  ZS_B3_ROUND(m, 9, 14, 11, 5, 8, 12, 15, 1, 13, 3, 0, 10, 2, 6, 4, 7)
  ZS_B3_ROUND(m, 11, 15, 5, 0, 1, 9, 8, 6, 14, 10, 2, 12, 3, 4, 7, 13)
  out[0] = v0 ^ v8;
  out[1] = v1 ^ v9;
  out[2] = v2 ^ v10;
  out[3] = v3 ^ v11;
  out[4] = v4 ^ v12;
  out[5] = v5 ^ v13;
  out[6] = v6 ^ v14;
  out[7] = v7 ^ v15;
  out[8] = v8 ^ cv[0];
  out[9] = v9 ^ cv[1];
  out[10] = v10 ^ cv[2];
  out[11] = v11 ^ cv[3];
  out[12] = v12 ^ cv[4];
  out[13] = v13 ^ cv[5];
  out[14] = v14 ^ cv[6];
  out[15] = v15 ^ cv[7];
}

#ifdef __CUDA_ARCH__
// compress_full with the rounds in a loop and the message permuted between rounds
// (m'[i] = m[PERM[i]], PERM = 2 6 3 10 7 0 4 13 1 11 12 5 9 14 15 8), not inlined:
// a few hundred bytes of code instead of several kilobytes per inlined copy. The
// device transcript runs in one thread per kernel, often with cold caches, where
// fetching unrolled code costs more than the rounds.
static __device__ __noinline__ void compress_rolled(const uint32_t cv[8], const uint32_t m_in[16],
                                                    uint64_t counter, uint32_t block_len, uint32_t flags,
                                                    uint32_t out[16]) {
  uint32_t m[16];
  for (int i = 0; i < 16; ++i) m[i] = m_in[i];
  uint32_t v0 = cv[0], v1 = cv[1], v2 = cv[2], v3 = cv[3], v4 = cv[4], v5 = cv[5], v6 = cv[6], v7 = cv[7];
  uint32_t v8 = IV0, v9 = IV1, v10 = IV2, v11 = IV3;
  uint32_t v12 = (uint32_t)counter, v13 = (uint32_t)(counter >> 32), v14 = block_len, v15 = flags;
#pragma unroll 1
  for (int r = 0; r < 7; ++r) {
    ZS_B3_ROUND(m, 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15)
    const uint32_t t0 = m[2], t1 = m[6], t2 = m[3], t3 = m[10], t4 = m[7], t5 = m[0], t6 = m[4], t7 = m[13];
    const uint32_t t8 = m[1], t9 = m[11], t10 = m[12], t11 = m[5], t12 = m[9], t13 = m[14], t14 = m[15], t15 = m[8];
    m[0] = t0, m[1] = t1, m[2] = t2, m[3] = t3, m[4] = t4, m[5] = t5, m[6] = t6, m[7] = t7;
    m[8] = t8, m[9] = t9, m[10] = t10, m[11] = t11, m[12] = t12, m[13] = t13, m[14] = t14, m[15] = t15;
  }
  out[0] = v0 ^ v8, out[1] = v1 ^ v9, out[2] = v2 ^ v10, out[3] = v3 ^ v11;
  out[4] = v4 ^ v12, out[5] = v5 ^ v13, out[6] = v6 ^ v14, out[7] = v7 ^ v15;
  out[8] = v8 ^ cv[0], out[9] = v9 ^ cv[1], out[10] = v10 ^ cv[2], out[11] = v11 ^ cv[3];
  out[12] = v12 ^ cv[4], out[13] = v13 ^ cv[5], out[14] = v14 ^ cv[6], out[15] = v15 ^ cv[7];
}
#endif
// The transcript's compression: unrolled on the host, compress_rolled on the device.
ZS_HD void compress_tx(const uint32_t cv[8], const uint32_t m[16], uint64_t counter, uint32_t block_len,
                       uint32_t flags, uint32_t out[16]) {
#ifdef __CUDA_ARCH__
  compress_rolled(cv, m, counter, block_len, flags, out);
#else
  compress_full(cv, m, counter, block_len, flags, out);
#endif
}

ZS_HD void iv(uint32_t cv[8]) {
  cv[0] = IV0; cv[1] = IV1; cv[2] = IV2; cv[3] = IV3;
  cv[4] = IV4; cv[5] = IV5; cv[6] = IV6; cv[7] = IV7;
}

// hashQM31 (src/m31/hash.zig:33-37): Blake3 of the 16-byte LE encoding, one
// compression with CHUNK_START | CHUNK_END | ROOT.
ZS_HD void hash_qm31(const qm31& v, uint32_t out[8]) {
  uint32_t m[16] = {v.a.a, v.a.b, v.b.a, v.b.b, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  iv(out);
  compress_cv(out, m, 16, CHUNK_START | CHUNK_END | ROOT);
}

// hash2 (src/core/hash/hash.zig:17-25): Blake3("zig-stark:pair" || L || R), 78 bytes
// in two blocks: block 0 = 14 prefix bytes + L + 18 bytes of R, block 1 = the last
// 14 bytes of R. Words are little-endian.
ZS_HD void hash2(const uint32_t l[8], const uint32_t r[8], uint32_t out[8]) {
  // "zig-stark:pair" = 7a 69 67 2d 73 74 61 72 6b 3a 70 61 69 72
  uint32_t m[16];
  m[0] = 0x2d67697au;  // "zig-"
  m[1] = 0x72617473u;  // "star"
  m[2] = 0x61703a6bu;  // "k:pa"
  // bytes 12,13 = "ir"; then L starts at byte 14 (2 bytes into word 3)
  m[3] = 0x00007269u | (l[0] << 16);
#pragma unroll
  for (int k = 1; k < 8; ++k) m[3 + k] = (l[k - 1] >> 16) | (l[k] << 16);
  // word 11 holds the last 2 bytes of L and the first 2 of R
  m[11] = (l[7] >> 16) | (r[0] << 16);
#pragma unroll
  for (int k = 1; k < 5; ++k) m[11 + k] = (r[k - 1] >> 16) | (r[k] << 16);
  iv(out);
  compress_cv(out, m, 64, CHUNK_START);
  // block 1: bytes 64..77 = R bytes 18..31 (14 bytes), zero padded
  uint32_t m2[16];
  m2[0] = (r[4] >> 16) | (r[5] << 16);
  m2[1] = (r[5] >> 16) | (r[6] << 16);
  m2[2] = (r[6] >> 16) | (r[7] << 16);
  m2[3] = r[7] >> 16;
#pragma unroll
  for (int k = 4; k < 16; ++k) m2[k] = 0;
  compress_cv(out, m2, 14, CHUNK_END | ROOT);
}

// Blake3 of a single-chunk message given as `nwords` little-endian u32 words
// (nwords * 4 <= 1024), e.g. hashM31s over a row (src/m31/hash.zig:15-25).
template <typename Loader>
ZS_HD void hash_words(int nwords, Loader load, uint32_t out[8]) {
  iv(out);
  int nblocks = (nwords * 4 + 63) / 64;
  if (nblocks == 0) nblocks = 1;
  for (int blk = 0; blk < nblocks; ++blk) {
    uint32_t m[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      int w = blk * 16 + k;
      m[k] = w < nwords ? load(w) : 0u;
    }
    int rem = nwords * 4 - blk * 64;
    uint32_t len = rem >= 64 ? 64u : (uint32_t)rem;
    uint32_t flags = (blk == 0 ? CHUNK_START : 0) | (blk == nblocks - 1 ? (CHUNK_END | ROOT) : 0);
    compress_cv(out, m, len, flags);
  }
}

}  // namespace b3

// Incremental Blake3 over arbitrary lengths (chunk state plus the chaining-value
// stack) for the transcript, on the host and, in one thread, on the device. Copyable,
// so the transcript can be snapshotted; snapshot_from copies only the live stack.
ZS_HD void copy_bytes(void* dst, const void* src, size_t n) {
  uint8_t* d = static_cast<uint8_t*>(dst);
  const uint8_t* s = static_cast<const uint8_t*>(src);
  for (size_t i = 0; i < n; ++i) d[i] = s[i];
}

struct Hasher {
  uint32_t cv[8];
  uint64_t chunk_counter = 0;
  uint8_t block[64];
  uint32_t block_len = 0, blocks_done = 0;
  uint32_t stack[54][8];
  unsigned depth = 0;

  ZS_HD Hasher() { reset(); }
  ZS_HD void reset() {
    b3::iv(cv);
    chunk_counter = 0;
    for (int i = 0; i < 64; ++i) block[i] = 0;
    block_len = blocks_done = 0;
    depth = 0;
  }
  ZS_HD void snapshot_from(const Hasher& o) {
    copy_bytes(cv, o.cv, 32);
    chunk_counter = o.chunk_counter;
    copy_bytes(block, o.block, 64);
    block_len = o.block_len;
    blocks_done = o.blocks_done;
    depth = o.depth;
    copy_bytes(stack, o.stack, (size_t)32 * o.depth);
  }
  ZS_HD static void words(const uint8_t* b, uint32_t w[16]) {
    for (int i = 0; i < 16; ++i)
      w[i] = (uint32_t)b[4 * i] | ((uint32_t)b[4 * i + 1] << 8) | ((uint32_t)b[4 * i + 2] << 16) |
             ((uint32_t)b[4 * i + 3] << 24);
  }
  ZS_HD uint32_t start() const { return blocks_done == 0 ? b3::CHUNK_START : 0; }
  ZS_HD void push(uint32_t c[8], uint64_t total) {
    while ((total & 1) == 0) {
      uint32_t m[16], out[16];
      copy_bytes(m, stack[--depth], 32);
      copy_bytes(m + 8, c, 32);
      uint32_t k[8];
      b3::iv(k);
      b3::compress_tx(k, m, 0, 64, b3::PARENT, out);
      copy_bytes(c, out, 32);
      total >>= 1;
    }
    copy_bytes(stack[depth++], c, 32);
  }
  ZS_HD void update(const void* data, size_t len) {
    const uint8_t* in = (const uint8_t*)data;
    while (len) {
      if (blocks_done * 64 + block_len == 1024) {
        uint32_t m[16], out[16];
        words(block, m);
        b3::compress_tx(cv, m, chunk_counter, block_len, start() | b3::CHUNK_END, out);
        ++chunk_counter;
        push(out, chunk_counter);
        b3::iv(cv);
        for (int i = 0; i < 64; ++i) block[i] = 0;
        block_len = blocks_done = 0;
      }
      if (block_len == 64) {
        uint32_t m[16], out[16];
        words(block, m);
        b3::compress_tx(cv, m, chunk_counter, 64, start(), out);
        copy_bytes(cv, out, 32);
        ++blocks_done;
        for (int i = 0; i < 64; ++i) block[i] = 0;
        block_len = 0;
      }
      size_t take = 64 - block_len;
      if (take > len) take = len;
      copy_bytes(block + block_len, in, take);
      block_len += (uint32_t)take;
      in += take;
      len -= take;
    }
  }
  ZS_HD void finalize(uint8_t out32[32]) const {
    uint32_t m[16], out[16];
    words(block, m);
    uint32_t flags = start() | b3::CHUNK_END;
    if (depth == 0) {
      b3::compress_tx(cv, m, chunk_counter, block_len, flags | b3::ROOT, out);
    } else {
      b3::compress_tx(cv, m, chunk_counter, block_len, flags, out);
      for (unsigned k = depth; k-- > 0;) {
        uint32_t pm[16], key[8];
        copy_bytes(pm, stack[k], 32);
        copy_bytes(pm + 8, out, 32);
        b3::iv(key);
        b3::compress_tx(key, pm, 0, 64, b3::PARENT | (k == 0 ? b3::ROOT : 0), out);
      }
    }
    for (int i = 0; i < 8; ++i) {
      out32[4 * i] = (uint8_t)out[i];
      out32[4 * i + 1] = (uint8_t)(out[i] >> 8);
      out32[4 * i + 2] = (uint8_t)(out[i] >> 16);
      out32[4 * i + 3] = (uint8_t)(out[i] >> 24);
    }
  }
  // finalize() of the state followed by `n` <= 64 more bytes, state unchanged, without
  // a snapshot: the chunk state is copied into words, the stack read in place, and a
  // chunk finished by the suffix (at most one) becomes a virtual top of the stack.
  ZS_HD void finalize_suffix(const uint8_t* suf, unsigned n, uint32_t o[8]) const {
    uint32_t c[8], m[16], out[16], top[8];
    for (int i = 0; i < 8; ++i) c[i] = cv[i];
    words(block, m);
    uint32_t len = block_len, blocks = blocks_done;
    uint64_t counter = chunk_counter;
    unsigned d = depth;
    bool has_top = false;
    for (unsigned i = 0; i < n; ++i) {
      if (blocks * 64 + len == 1024) {  // chunk full: its chaining value goes on the stack
        b3::compress_tx(c, m, counter, len, (blocks == 0 ? b3::CHUNK_START : 0) | b3::CHUNK_END, out);
        for (int w = 0; w < 8; ++w) top[w] = out[w];
        for (uint64_t total = counter + 1; (total & 1) == 0; total >>= 1) {
          uint32_t pm[16], key[8];
          for (int w = 0; w < 8; ++w) pm[w] = stack[d - 1][w], pm[8 + w] = top[w];
          b3::iv(key);
          b3::compress_tx(key, pm, 0, 64, b3::PARENT, out);
          for (int w = 0; w < 8; ++w) top[w] = out[w];
          --d;
        }
        has_top = true;
        b3::iv(c);
        for (int w = 0; w < 16; ++w) m[w] = 0;
        len = blocks = 0;
        ++counter;
      } else if (len == 64) {
        b3::compress_tx(c, m, counter, 64, blocks == 0 ? b3::CHUNK_START : 0, out);
        for (int w = 0; w < 8; ++w) c[w] = out[w];
        for (int w = 0; w < 16; ++w) m[w] = 0;
        len = 0;
        ++blocks;
      }
      m[len >> 2] |= (uint32_t)suf[i] << (8 * (len & 3));
      ++len;
    }
    const unsigned total = d + (has_top ? 1u : 0u);
    const uint32_t flags = (blocks == 0 ? b3::CHUNK_START : 0) | b3::CHUNK_END;
    b3::compress_tx(c, m, counter, len, flags | (total == 0 ? b3::ROOT : 0), out);
    for (int w = 0; w < 8; ++w) o[w] = out[w];
    for (unsigned k = total; k-- > 0;) {
      uint32_t pm[16], key[8];
      const uint32_t* l = has_top && k == d ? top : stack[k];
      for (int w = 0; w < 8; ++w) pm[w] = l[w], pm[8 + w] = o[w];
      b3::iv(key);
      b3::compress_tx(key, pm, 0, 64, b3::PARENT | (k == 0 ? b3::ROOT : 0), out);
      for (int w = 0; w < 8; ++w) o[w] = out[w];
    }
  }
};

}  // namespace zs
