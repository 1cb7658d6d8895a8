// ORACLE — test infrastructure only. The Binius tower field and the per-round
// sum-check evaluation, restated from:
//   src/binius/tower.zig      TowerField(level): fromInt 52-56, add 58-60, betaValue 45-50,
//                             mulRec 228-248 (Karatsuba over the subfield,
//                             hi = (c2 + c0 + c1) + c1·β), alpha 314-317
//   src/binius/sumcheck.zig   proveCombinationWith 357-372: the single-threaded
//                             values[t] loop, points[t] = fromInt(t)
//   src/binius/accel.zig      9-26, 43-47: the flattened inputs the GPU hook takes
//   src/binius/sumcheck.zig   Transcript 47-87 (SHA-256), runRounds 97-121,
//                             interpolateCoeffs 124-162, evalPoly 164-172,
//                             computeCombinationSum 187-200, proveCombinationWith 232-395
//                             (the CPU path; the fold of every table after each round)
//   src/binius/polynomial.zig Multilinear.eval 35-51 (the same fold, lowest variable first)
//   src/binius/tower.zig      toBytes / fromBytes 334-350 (little-endian, SIZE bytes)
// Elements are the tower's bit strings (level L: the low 2^L bits of a u128).
#pragma once
#include <algorithm>
#include <array>
#include <cstdint>
#include <cstring>
#include <optional>
#include <stdexcept>
#include <vector>

namespace orc {

using u128 = unsigned __int128;

inline unsigned towerBits(unsigned level) { return 1u << level; }
inline u128 towerMask(unsigned level) { return level >= 7 ? ~(u128)0 : (((u128)1 << towerBits(level)) - 1); }

// betaValue (tower.zig:45-50): 0 at level 0, 1 at level 1, X_{level-2} above.
inline u128 towerBeta(unsigned level) {
  if (level == 0) return 0;
  if (level == 1) return 1;
  return (u128)1 << (1u << (level - 2));
}

// mulRec (tower.zig:228-248).
inline u128 towerMul(unsigned level, u128 a, u128 b) {
  if (level == 0) return a & b & 1;
  const unsigned half = 1u << (level - 1);
  const u128 mask = ((u128)1 << half) - 1;
  const u128 a0 = a & mask, a1 = (a >> half) & mask, b0 = b & mask, b1 = (b >> half) & mask;
  const u128 c0 = towerMul(level - 1, a0, b0);
  const u128 c1 = towerMul(level - 1, a1, b1);
  const u128 c2 = towerMul(level - 1, a0 ^ a1, b0 ^ b1);
  const u128 lo = c0 ^ c1;
  const u128 hi = c2 ^ c0 ^ c1 ^ towerMul(level - 1, c1, towerBeta(level));
  return lo | (hi << half);
}

// One round's values[t], t = 0..dmax (sumcheck.zig:357-372), over TowerField(level):
// cur[f][i] for f < m, i < len (len = 2 half); term k multiplies coeffs[k] by the factors
// indices[offsets[k] .. offsets[k+1]).
inline std::vector<u128> sumcheckRoundValues(unsigned level, const std::vector<std::vector<u128>>& cur,
                                             const std::vector<u128>& coeffs, const std::vector<uint32_t>& indices,
                                             const std::vector<uint32_t>& offsets, size_t dmax, size_t half) {
  std::vector<u128> values(dmax + 1, 0);
  const u128 mask = towerMask(level);
  for (size_t t = 0; t <= dmax; ++t) {
    const u128 point = (u128)t & mask;  // fromInt(t)
    u128 s = 0;
    for (size_t rest = 0; rest < half; ++rest) {
      for (size_t k = 0; k < coeffs.size(); ++k) {
        u128 prod = coeffs[k];
        for (uint32_t j = offsets[k]; j < offsets[k + 1]; ++j) {
          const u128 a = cur[indices[j]][2 * rest], b = cur[indices[j]][2 * rest + 1];
          prod = towerMul(level, prod, a ^ towerMul(level, point, a ^ b));
        }
        s ^= prod;
      }
    }
    values[t] = s;
  }
  return values;
}

// ---- SHA-256 (FIPS 180-4): std.crypto.hash.sha2.Sha256 of the transcript ----------

inline std::array<uint8_t, 32> sha256(const uint8_t* msg, size_t n) {
  static const uint32_t K[64] = {
      0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5,
      0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174,
      0xe49b69c1, 0xefbe4786, 0x0fc19dc6, 0x240ca1cc, 0x2de92c6f, 0x4a7484aa, 0x5cb0a9dc, 0x76f988da,
      0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7, 0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967,
      0x27b70a85, 0x2e1b2138, 0x4d2c6dfc, 0x53380d13, 0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85,
      0xa2bfe8a1, 0xa81a664b, 0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070,
      0x19a4c116, 0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a, 0x5b9cca4f, 0x682e6ff3,
      0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7, 0xc67178f2};
  // the padded message: msg, 0x80, zeros to 56 mod 64, the bit length big-endian
  std::vector<uint8_t> m(msg, msg + n);
  m.push_back(0x80);
  while (m.size() % 64 != 56) m.push_back(0);
  for (int i = 7; i >= 0; --i) m.push_back((uint8_t)(((uint64_t)n * 8) >> (8 * i)));
  uint32_t H[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a, 0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};
  auto rotr = [](uint32_t x, int r) { return (x >> r) | (x << (32 - r)); };
  for (size_t off = 0; off < m.size(); off += 64) {
    uint32_t W[64];
    for (int t = 0; t < 16; ++t) {
      W[t] = 0;
      for (int b = 0; b < 4; ++b) W[t] = (W[t] << 8) | m[off + 4 * t + b];
    }
    for (int t = 16; t < 64; ++t) {
      const uint32_t x = W[t - 15], y = W[t - 2];
      W[t] = (rotr(y, 17) ^ rotr(y, 19) ^ (y >> 10)) + W[t - 7] + (rotr(x, 7) ^ rotr(x, 18) ^ (x >> 3)) + W[t - 16];
    }
    uint32_t v[8];
    for (int i = 0; i < 8; ++i) v[i] = H[i];
    for (int t = 0; t < 64; ++t) {
      const uint32_t T1 = v[7] + (rotr(v[4], 6) ^ rotr(v[4], 11) ^ rotr(v[4], 25)) + ((v[4] & v[5]) ^ (~v[4] & v[6])) +
                          K[t] + W[t];
      const uint32_t T2 = (rotr(v[0], 2) ^ rotr(v[0], 13) ^ rotr(v[0], 22)) + ((v[0] & v[1]) ^ (v[0] & v[2]) ^ (v[1] & v[2]));
      for (int i = 7; i > 0; --i) v[i] = v[i - 1];
      v[4] += T1;
      v[0] = T1 + T2;
    }
    for (int i = 0; i < 8; ++i) H[i] += v[i];
  }
  std::array<uint8_t, 32> out;
  for (int i = 0; i < 32; ++i) out[i] = (uint8_t)(H[i / 4] >> (24 - 8 * (i % 4)));
  return out;
}

// ---- the sum-check prover and verifier over TowerField(level) ---------------------

inline size_t towerSize(unsigned level) { return ((1u << level) + 7) / 8; }

inline void towerToBytes(unsigned level, u128 v, uint8_t* out) {
  for (size_t i = 0; i < towerSize(level); ++i) out[i] = (uint8_t)(v >> (8 * i));
}
inline u128 towerFromBytes(unsigned level, const uint8_t* p) {
  u128 v = 0;
  for (size_t i = towerSize(level); i-- > 0;) v = (v << 8) | p[i];
  return v & towerMask(level);
}

// a^(2^BITS - 2) = a^-1 (a != 0): BITS - 1 squarings, each multiplied into the result.
inline u128 towerInv(unsigned level, u128 a) {
  u128 r = 1, x = a;
  for (unsigned i = 1; i < towerBits(level); ++i) {
    x = towerMul(level, x, x);
    r = towerMul(level, r, x);
  }
  return r;
}

struct SumcheckTranscript {
  unsigned level;
  std::array<uint8_t, 32> buf;
  static SumcheckTranscript init(unsigned level, u128 claimed) {
    uint8_t b[16];
    towerToBytes(level, claimed, b);
    return {level, sha256(b, towerSize(level))};
  }
  static SumcheckTranscript initBytes(unsigned level, const std::vector<uint8_t>& seed) {
    return {level, sha256(seed.data(), seed.size())};
  }
  u128 absorb(const std::vector<u128>& coeffs) {
    std::vector<uint8_t> msg(buf.begin(), buf.end());
    uint8_t b[16];
    for (u128 c : coeffs) {
      towerToBytes(level, c, b);
      msg.insert(msg.end(), b, b + towerSize(level));
    }
    buf = sha256(msg.data(), msg.size());
    if (towerSize(level) == 1) return (u128)buf[31] & towerMask(level);
    return towerFromBytes(level, buf.data() + 32 - towerSize(level));
  }
};

inline std::vector<u128> interpolateCoeffs(unsigned level, const std::vector<u128>& points,
                                           const std::vector<u128>& values) {
  const size_t n = points.size();
  std::vector<u128> coeffs(n, 0);
  for (size_t i = 0; i < n; ++i) {
    std::vector<u128> basis{1};
    u128 denom = 1;
    for (size_t j = 0; j < n; ++j) {
      if (j == i) continue;
      std::vector<u128> next(basis.size() + 1, 0);  // basis * (t + points[j])
      for (size_t d = 0; d < basis.size(); ++d) {
        next[d + 1] ^= basis[d];
        next[d] ^= towerMul(level, points[j], basis[d]);
      }
      basis = next;
      denom = towerMul(level, denom, points[i] ^ points[j]);
    }
    const u128 scale = towerMul(level, towerInv(level, denom), values[i]);
    for (size_t d = 0; d < basis.size(); ++d) coeffs[d] ^= towerMul(level, basis[d], scale);
  }
  return coeffs;
}

inline u128 evalPoly(unsigned level, const std::vector<u128>& coeffs, u128 x) {
  u128 acc = 0;
  for (size_t i = coeffs.size(); i-- > 0;) acc = towerMul(level, acc, x) ^ coeffs[i];
  return acc;
}

// cur[f][rest] = a + r (a + b) for rest < len / 2: the fold after each round and
// Multilinear.eval's step.
inline void foldTables(unsigned level, std::vector<std::vector<u128>>& cur, size_t len, u128 r) {
  for (auto& ct : cur)
    for (size_t rest = 0; rest < len / 2; ++rest) {
      const u128 a = ct[2 * rest], b = ct[2 * rest + 1];
      ct[rest] = a ^ towerMul(level, r, a ^ b);
    }
}

struct SumcheckTerms {
  std::vector<u128> coeffs;
  std::vector<uint32_t> indices, offsets;
  size_t dmax() const {
    size_t d = 0;
    for (size_t k = 0; k + 1 < offsets.size(); ++k) d = std::max<size_t>(d, offsets[k + 1] - offsets[k]);
    return d;
  }
};

struct SumcheckProof {
  u128 claimed;
  std::vector<std::vector<u128>> rounds;
};

inline u128 combinationAt(unsigned level, const std::vector<std::vector<u128>>& tables, const SumcheckTerms& tm,
                          size_t idx) {
  u128 s = 0;
  for (size_t k = 0; k < tm.coeffs.size(); ++k) {
    u128 prod = tm.coeffs[k];
    for (uint32_t j = tm.offsets[k]; j < tm.offsets[k + 1]; ++j) prod = towerMul(level, prod, tables[tm.indices[j]][idx]);
    s ^= prod;
  }
  return s;
}

inline SumcheckProof proveCombination(unsigned level, size_t k, const std::vector<std::vector<u128>>& tables,
                                      const SumcheckTerms& tm, const std::vector<uint8_t>* seed) {
  const size_t n = (size_t)1 << k, dmax = tm.dmax();
  u128 h = 0;
  for (size_t x = 0; x < n; ++x) h ^= combinationAt(level, tables, tm, x);
  SumcheckTranscript tr = seed ? SumcheckTranscript::initBytes(level, *seed) : SumcheckTranscript::init(level, h);
  std::vector<std::vector<u128>> cur = tables;
  std::vector<u128> points(dmax + 1);
  for (size_t t = 0; t <= dmax; ++t) points[t] = (u128)t & towerMask(level);
  SumcheckProof pf{h, {}};
  size_t len = n;
  for (size_t i = 0; i < k; ++i) {
    const size_t half = len / 2;
    const std::vector<u128> values = sumcheckRoundValues(level, cur, tm.coeffs, tm.indices, tm.offsets, dmax, half);
    pf.rounds.push_back(interpolateCoeffs(level, points, values));
    const u128 r = tr.absorb(pf.rounds.back());
    foldTables(level, cur, len, r);
    len = half;
  }
  return pf;
}

// runRounds: s_i(0) + s_i(1) = the running sum, the challenges, the final running sum.
inline std::optional<std::pair<std::vector<u128>, u128>> runRounds(unsigned level, const std::vector<uint8_t>* seed,
                                                                   u128 claimed,
                                                                   const std::vector<std::vector<u128>>& rounds) {
  SumcheckTranscript tr = seed ? SumcheckTranscript::initBytes(level, *seed) : SumcheckTranscript::init(level, claimed);
  std::vector<u128> ch;
  u128 cur = claimed;
  for (const auto& cs : rounds) {
    if ((evalPoly(level, cs, 0) ^ evalPoly(level, cs, 1)) != cur) return std::nullopt;
    const u128 r = tr.absorb(cs);
    ch.push_back(r);
    cur = evalPoly(level, cs, r);
  }
  return std::make_pair(ch, cur);
}

inline u128 multilinearEval(unsigned level, std::vector<u128> table, const std::vector<u128>& r) {
  std::vector<std::vector<u128>> one{std::move(table)};
  size_t len = one[0].size();
  for (u128 ri : r) {
    foldTables(level, one, len, ri);
    len /= 2;
  }
  return one[0][0];
}

// The combination round trip of sumcheck.zig:632-665: the rounds replay, and the final
// running sum is g at the challenge point, sum coeff * prod MLE_j(challenges).
inline bool verifyCombination(unsigned level, size_t k, const std::vector<std::vector<u128>>& tables,
                              const SumcheckTerms& tm, const SumcheckProof& pf, const std::vector<uint8_t>* seed) {
  if (pf.rounds.size() != k) return false;
  const auto rr = runRounds(level, seed, pf.claimed, pf.rounds);
  if (!rr) return false;
  std::vector<std::vector<u128>> ev(tables.size(), std::vector<u128>(1));
  for (size_t f = 0; f < tables.size(); ++f) ev[f][0] = multilinearEval(level, tables[f], rr->first);
  return combinationAt(level, ev, tm, 0) == rr->second;
}

}  // namespace orc
