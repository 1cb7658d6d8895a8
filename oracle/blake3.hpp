// ORACLE — test infrastructure only. BLAKE3 (unkeyed hash mode, 32-byte output)
// restated from the public BLAKE3 specification. The reference calls Zig 0.16.0
// `std.crypto.hash.Blake3` (src/core/hash/hash.zig:9-24, src/m31/hash.zig:16-24,
// src/core/channel/channel.zig:12-21,56-62), which is not vendored; this
// restatement is pinned by the reference's Blake3("") known answer
// (src/core/hash/hash.zig:32-43) and cross-checked against the `blake3` Python
// package in the tests for every input length the path uses.
//
// The hasher is a plain value type: copying it snapshots the transcript, which
// is how Channel.sampleBytes (channel.zig:56-62) derives challenge blocks.
#pragma once
#include <cstdint>
#include <cstring>

namespace orc {

namespace b3 {
constexpr uint32_t IV[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                            0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};
constexpr unsigned PERM[16] = {2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8};
constexpr uint32_t CHUNK_START = 1, CHUNK_END = 2, PARENT = 4, ROOT = 8;
constexpr size_t BLOCK_LEN = 64, CHUNK_LEN = 1024;

inline uint32_t rotr(uint32_t x, unsigned n) { return (x >> n) | (x << (32 - n)); }

inline void g(uint32_t* s, int a, int b, int c, int d, uint32_t mx, uint32_t my) {
  s[a] = s[a] + s[b] + mx;
  s[d] = rotr(s[d] ^ s[a], 16);
  s[c] = s[c] + s[d];
  s[b] = rotr(s[b] ^ s[c], 12);
  s[a] = s[a] + s[b] + my;
  s[d] = rotr(s[d] ^ s[a], 8);
  s[c] = s[c] + s[d];
  s[b] = rotr(s[b] ^ s[c], 7);
}

// The compression function: returns the full 16-word output state.
inline void compress(const uint32_t cv[8], const uint32_t block[16], uint64_t counter,
                     uint32_t block_len, uint32_t flags, uint32_t out[16]) {
  uint32_t s[16] = {cv[0], cv[1], cv[2], cv[3], cv[4], cv[5], cv[6], cv[7],
                    IV[0], IV[1], IV[2], IV[3], (uint32_t)counter, (uint32_t)(counter >> 32),
                    block_len, flags};
  uint32_t m[16];
  std::memcpy(m, block, 64);
  for (int r = 0; r < 7; ++r) {
    g(s, 0, 4, 8, 12, m[0], m[1]);
    g(s, 1, 5, 9, 13, m[2], m[3]);
    g(s, 2, 6, 10, 14, m[4], m[5]);
    g(s, 3, 7, 11, 15, m[6], m[7]);
    g(s, 0, 5, 10, 15, m[8], m[9]);
    g(s, 1, 6, 11, 12, m[10], m[11]);
    g(s, 2, 7, 8, 13, m[12], m[13]);
    g(s, 3, 4, 9, 14, m[14], m[15]);
    if (r < 6) {
      uint32_t t[16];
      for (int i = 0; i < 16; ++i) t[i] = m[PERM[i]];
      std::memcpy(m, t, 64);
    }
  }
  for (int i = 0; i < 8; ++i) {
    out[i] = s[i] ^ s[i + 8];
    out[i + 8] = s[i + 8] ^ cv[i];
  }
}

inline void wordsFromBytes(const uint8_t* b, uint32_t w[16]) {
  for (int i = 0; i < 16; ++i)
    w[i] = (uint32_t)b[4 * i] | ((uint32_t)b[4 * i + 1] << 8) | ((uint32_t)b[4 * i + 2] << 16) |
           ((uint32_t)b[4 * i + 3] << 24);
}
}  // namespace b3

// Incremental BLAKE3 hasher (chunk state + chaining-value stack).
struct Blake3 {
  // current chunk
  uint32_t cv[8];
  uint64_t chunk_counter = 0;
  uint8_t block[64];
  uint32_t block_len = 0;
  uint32_t blocks_compressed = 0;
  // stack of completed subtree chaining values
  uint32_t stack[54][8];
  unsigned stack_len = 0;

  Blake3() { reset(); }
  void reset() {
    std::memcpy(cv, b3::IV, 32);
    chunk_counter = 0;
    std::memset(block, 0, 64);
    block_len = 0;
    blocks_compressed = 0;
    stack_len = 0;
  }

  uint32_t startFlag() const { return blocks_compressed == 0 ? b3::CHUNK_START : 0; }
  size_t chunkLen() const { return b3::BLOCK_LEN * blocks_compressed + block_len; }

  void pushCv(const uint32_t newcv[8], uint64_t total_chunks) {
    uint32_t cur[8];
    std::memcpy(cur, newcv, 32);
    // Merge completed subtrees: one merge per trailing zero of total_chunks.
    while ((total_chunks & 1) == 0) {
      uint32_t blockw[16], out[16];
      std::memcpy(blockw, stack[stack_len - 1], 32);
      std::memcpy(blockw + 8, cur, 32);
      --stack_len;
      b3::compress(b3::IV, blockw, 0, 64, b3::PARENT, out);
      std::memcpy(cur, out, 32);
      total_chunks >>= 1;
    }
    std::memcpy(stack[stack_len++], cur, 32);
  }

  void update(const void* data, size_t len) {
    const uint8_t* in = (const uint8_t*)data;
    while (len > 0) {
      if (chunkLen() == b3::CHUNK_LEN) {
        // The chunk is full and more input follows: finish it as a non-root chunk.
        uint32_t w[16], out[16];
        b3::wordsFromBytes(block, w);
        b3::compress(cv, w, chunk_counter, block_len, startFlag() | b3::CHUNK_END, out);
        uint64_t total = chunk_counter + 1;
        pushCv(out, total);
        std::memcpy(cv, b3::IV, 32);
        chunk_counter = total;
        std::memset(block, 0, 64);
        block_len = 0;
        blocks_compressed = 0;
      }
      if (block_len == b3::BLOCK_LEN) {
        uint32_t w[16], out[16];
        b3::wordsFromBytes(block, w);
        b3::compress(cv, w, chunk_counter, 64, startFlag(), out);
        std::memcpy(cv, out, 32);
        ++blocks_compressed;
        std::memset(block, 0, 64);
        block_len = 0;
      }
      size_t want = b3::BLOCK_LEN - block_len;
      size_t take = want < len ? want : len;
      std::memcpy(block + block_len, in, take);
      block_len += (uint32_t)take;
      in += take;
      len -= take;
    }
  }

  // 32-byte root output; does not modify the hasher.
  void finalize(uint8_t out32[32]) const {
    uint32_t w[16], out[16];
    b3::wordsFromBytes(block, w);
    uint32_t flags = startFlag() | b3::CHUNK_END;
    if (stack_len == 0) {
      b3::compress(cv, w, chunk_counter, block_len, flags | b3::ROOT, out);
    } else {
      b3::compress(cv, w, chunk_counter, block_len, flags, out);
      uint32_t cur[8];
      std::memcpy(cur, out, 32);
      for (unsigned k = stack_len; k-- > 0;) {
        uint32_t blockw[16];
        std::memcpy(blockw, stack[k], 32);
        std::memcpy(blockw + 8, cur, 32);
        uint32_t f = b3::PARENT | (k == 0 ? b3::ROOT : 0);
        b3::compress(b3::IV, blockw, 0, 64, f, out);
        std::memcpy(cur, out, 32);
      }
    }
    for (int i = 0; i < 8; ++i) {
      out32[4 * i] = (uint8_t)out[i];
      out32[4 * i + 1] = (uint8_t)(out[i] >> 8);
      out32[4 * i + 2] = (uint8_t)(out[i] >> 16);
      out32[4 * i + 3] = (uint8_t)(out[i] >> 24);
    }
  }
};

inline void blake3Hash(const void* data, size_t len, uint8_t out32[32]) {
  Blake3 h;
  h.update(data, len);
  h.finalize(out32);
}

}  // namespace orc
