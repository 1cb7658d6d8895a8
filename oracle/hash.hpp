// ORACLE — test infrastructure only. Digests, Merkle trees and the Fiat-Shamir
// channel, restated from:
//   src/core/hash/hash.zig      hashBytes 11-15, hash2 17-25
//   src/m31/hash.zig            hashM31s 15-25, hashQM31 33-37
//   src/core/merkle/merkle.zig  init 17-45, root 47, open 57-68, verify 72-89
//   src/core/channel/channel.zig init 16-21, absorb 27-43, sampleBytes 49-69,
//                                sample 72-76, sampleIndex 79-101
#pragma once
#include <array>
#include <cstdint>
#include <cstring>
#include <vector>

#include "blake3.hpp"
#include "field.hpp"

namespace orc {

using Digest = std::array<uint8_t, 32>;

inline Digest hashBytes(const void* msg, size_t len) {
  Digest d;
  blake3Hash(msg, len, d.data());
  return d;
}

// hash.zig:17-25: Blake3("zig-stark:pair" || a || b).
inline Digest hash2(const Digest& a, const Digest& b) {
  Blake3 h;
  h.update("zig-stark:pair", 14);
  h.update(a.data(), 32);
  h.update(b.data(), 32);
  Digest d;
  h.finalize(d.data());
  return d;
}

// m31/hash.zig:33-37: Blake3 of the 16-byte LE encoding.
inline Digest hashQM31(const QM31& v) {
  uint8_t buf[16];
  v.toBytes(buf);
  return hashBytes(buf, 16);
}

// m31/hash.zig:15-25: Blake3 of the concatenated 4-byte LE encodings.
inline Digest hashM31s(const M31* vals, size_t n) {
  Blake3 h;
  for (size_t i = 0; i < n; ++i) {
    uint8_t buf[4];
    vals[i].toBytes(buf);
    h.update(buf, 4);
  }
  Digest d;
  h.finalize(d.data());
  return d;
}

// merkle.zig:10-69. nodes[0] = leaves, nodes[depth] = {root}.
struct MerkleTree {
  std::vector<std::vector<Digest>> nodes;

  MerkleTree() = default;
  explicit MerkleTree(const std::vector<Digest>& leaves) { init(leaves); }

  void init(const std::vector<Digest>& leaves) {
    size_t n = leaves.size();
    // merkle.zig:19 power of two, n > 0
    unsigned depth = 0;
    while (((size_t)1 << depth) < n) ++depth;
    nodes.assign(depth + 1, {});
    nodes[0] = leaves;
    for (unsigned level = 0; level < depth; ++level) {
      size_t half = nodes[level].size() / 2;
      nodes[level + 1].resize(half);
      for (size_t i = 0; i < half; ++i)
        nodes[level + 1][i] = hash2(nodes[level][2 * i], nodes[level][2 * i + 1]);
    }
  }
  const Digest& root() const { return nodes.back()[0]; }
  size_t numLeaves() const { return nodes[0].size(); }
  // merkle.zig:57-68: siblings bottom-up.
  std::vector<Digest> open(size_t index) const {
    std::vector<Digest> path;
    size_t idx = index;
    for (size_t level = 0; level + 1 < nodes.size(); ++level) {
      path.push_back(nodes[level][idx ^ 1]);
      idx >>= 1;
    }
    return path;
  }
};

// merkle.zig:72-89.
inline bool merkleVerify(const Digest& root, size_t index, const Digest& leaf,
                         const std::vector<Digest>& path) {
  Digest d = leaf;
  size_t idx = index;
  for (const Digest& sib : path) {
    d = (idx & 1) == 0 ? hash2(d, sib) : hash2(sib, d);
    idx >>= 1;
  }
  return d == root;
}

// channel.zig:16-101.
struct Channel {
  Blake3 hasher;
  explicit Channel(const void* sep, size_t sep_len) {
    hasher.update("zig-stark:channel", 17);
    hasher.update(sep, sep_len);
  }
  void absorbBytes(const void* d, size_t n) { hasher.update(d, n); }
  void absorbDigest(const Digest& d) { hasher.update(d.data(), 32); }
  void absorb(const QM31& v) {
    uint8_t b[16];
    v.toBytes(b);
    hasher.update(b, 16);
  }
  void absorb(const M31& v) {
    uint8_t b[4];
    v.toBytes(b);
    hasher.update(b, 4);
  }
  void absorbMany(const std::vector<QM31>& vs) {
    for (const auto& v : vs) absorb(v);
  }
  // channel.zig:49-69: block k = Blake3(state || "zig-stark:sample" || u64le(k)),
  // each derived block is absorbed back into the transcript.
  void sampleBytes(uint8_t* out, size_t len) {
    uint64_t counter = 0;
    while (len > 0) {
      Blake3 snap = hasher;
      snap.update("zig-stark:sample", 16);
      uint8_t cb[8];
      for (int i = 0; i < 8; ++i) cb[i] = (uint8_t)(counter >> (8 * i));
      snap.update(cb, 8);
      uint8_t blk[32];
      snap.finalize(blk);
      hasher.update(blk, 32);
      size_t n = len < 32 ? len : 32;
      std::memcpy(out, blk, n);
      out += n;
      len -= n;
      ++counter;
    }
  }
  QM31 sampleQM31() {
    uint8_t b[16];
    sampleBytes(b, 16);
    return QM31::fromBytes(b);
  }
  M31 sampleM31() {
    uint8_t b[4];
    sampleBytes(b, 4);
    return M31::fromBytes(b);
  }
  // channel.zig:79-101: bits = log2(n) + 1, big-endian over ceil(bits/8) bytes,
  // masked, rejection-sampled into [0, n).
  uint64_t sampleIndex(uint64_t n) {
    unsigned lg = 0;
    while ((n >> (lg + 1)) != 0) ++lg;
    unsigned bits = lg + 1;
    unsigned nbytes = (bits + 7) / 8;
    uint64_t mask = bits >= 64 ? ~0ull : (((uint64_t)1 << bits) - 1);
    for (;;) {
      uint8_t buf[8];
      sampleBytes(buf, nbytes);
      uint64_t value = 0;
      for (unsigned i = 0; i < nbytes; ++i) value = (value << 8) | buf[i];
      uint64_t v = value & mask;
      if (v < n) return v;
    }
  }
};

}  // namespace orc
