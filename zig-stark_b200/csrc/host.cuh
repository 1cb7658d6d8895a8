// Host-side protocol pieces of the prover: the wire codec
// (src/core/serialization.zig:58-190), the Fiat-Shamir channel
// (src/core/channel/channel.zig:16-101) and small exact helpers. These run once per
// proof on a few hundred bytes; the heavy work stays on the device.
#pragma once
#include <array>
#include <cstring>
#include <vector>

#include "blake3.cuh"
#include "common.cuh"

namespace zs {

using Digest = std::array<uint8_t, 32>;

struct WireWriter {
  std::vector<uint8_t> out;
  // An unsigned integer of `width` bytes, little-endian (every int on the wire).
  void uint_le(uint64_t v, unsigned width) {
    for (unsigned i = 0; i < width; ++i) out.push_back((uint8_t)(v >> (8 * i)));
  }
  void u8(uint8_t v) { uint_le(v, 1); }
  void u64(uint64_t v) { uint_le(v, 8); }  // also every usize and slice length
  void flag(bool present) { u8(present ? 1 : 0); }  // bool, and an optional's presence byte
  void bytes(const void* p, size_t n) {
    const uint8_t* b = (const uint8_t*)p;
    out.insert(out.end(), b, b + n);
  }
  void digest(const Digest& d) { bytes(d.data(), 32); }
  void q(const qm31& v) {
    const uint32_t w[4] = {v.a.a, v.a.b, v.b.a, v.b.b};
    bytes(w, 16);
  }
  void digests(const std::vector<Digest>& v) {
    u64(v.size());
    for (auto& d : v) digest(d);
  }
  void qs(const std::vector<qm31>& v) {
    u64(v.size());
    for (auto& x : v) q(x);
  }
};

struct WireReader {
  const uint8_t* p;
  size_t n, pos = 0;
  WireReader(const uint8_t* d, size_t len) : p(d), n(len) {}
  const uint8_t* take(size_t k) {
    if (k > n - pos) throw Error(ZS_EMALFORMED, "unexpected end of input");
    const uint8_t* r = p + pos;
    pos += k;
    return r;
  }
  uint8_t u8() { return *take(1); }
  uint64_t u64() {
    const uint8_t* b = take(8);
    uint64_t v = 0;
    for (int i = 0; i < 8; ++i) v |= (uint64_t)b[i] << (8 * i);
    return v;
  }
  uint64_t len(size_t elem) {
    const uint64_t l = u64();
    if (elem && l > (n - pos) / elem) throw Error(ZS_EMALFORMED, "length prefix exceeds input");
    return l;
  }
  // M31.fromBytes reduces raw % p (m31.zig:97-100).
  static uint32_t m31(const uint8_t* b) {
    uint32_t r;
    std::memcpy(&r, b, 4);
    return r >= P ? r % P : r;
  }
  qm31 q() {
    const uint8_t* b = take(16);
    return qmake(m31(b), m31(b + 4), m31(b + 8), m31(b + 12));
  }
  void end() const {
    if (pos != n) throw Error(ZS_EMALFORMED, "trailing bytes");
  }
};

// StarkParams (stark.zig:75-90) and FriParams (fri.zig:38-55) on the wire:
// u8, u8, usize (8 bytes), u8.
struct StarkParamsH {
  uint8_t trace_log = 0, log_blowup = 3;
  uint64_t num_queries = 16;
  uint8_t remainder_log = 3;
};
struct FriParamsH {
  uint8_t log_size = 0, log_blowup = 3;
  uint64_t num_queries = 24;
  uint8_t remainder_log = 3;
  unsigned domain_log() const { return log_size + log_blowup; }
  unsigned folds() const { return domain_log() - remainder_log; }
};

// Fiat-Shamir channel (channel.zig): one running Blake3 over
// "zig-stark:channel" || separator || absorbed bytes; sample block k is
// Blake3(state || "zig-stark:sample" || u64le(k)) and is absorbed back. Usable on the
// host and, in one thread, on the device (the FRI commit phase runs its transcript
// steps there); the layout is the same on both sides, so the state is copied across.
ZS_HD uint32_t m31_from_le(const uint8_t* b) {  // M31.fromBytes (m31.zig:97-100)
  const uint32_t r = (uint32_t)b[0] | ((uint32_t)b[1] << 8) | ((uint32_t)b[2] << 16) | ((uint32_t)b[3] << 24);
  return r >= P ? r % P : r;
}

struct Channel {
  Hasher h;
  ZS_HD Channel(const void* sep, size_t n) {
    h.update("zig-stark:channel", 17);
    h.update(sep, n);
  }
  void absorb(const Digest& d) { h.update(d.data(), 32); }
  ZS_HD void absorb_bytes(const void* p, size_t n) { h.update(p, n); }
  ZS_HD void absorb(const qm31& v) {
    const uint32_t w[4] = {v.a.a, v.a.b, v.b.a, v.b.b};
    uint8_t b[16];
    for (int i = 0; i < 4; ++i)
      for (int k = 0; k < 4; ++k) b[4 * i + k] = (uint8_t)(w[i] >> (8 * k));
    h.update(b, 16);
  }
  // On the host a sample is drawn from a snapshot of the state (`scratch`, a local
  // copy when null); on the device, in one thread, from the state itself extended by
  // the suffix (Hasher::finalize_suffix), which copies no stack.
  ZS_HD void sample_bytes(uint8_t* out, size_t len, Hasher* scratch = nullptr) {
    uint64_t counter = 0;
    while (len) {
      uint8_t blk[32];
#ifdef __CUDA_ARCH__
      (void)scratch;
      uint8_t suf[24];
      copy_bytes(suf, "zig-stark:sample", 16);
      for (int i = 0; i < 8; ++i) suf[16 + i] = (uint8_t)(counter >> (8 * i));
      uint32_t o[8];
      h.finalize_suffix(suf, 24, o);
      for (int i = 0; i < 32; ++i) blk[i] = (uint8_t)(o[i / 4] >> (8 * (i % 4)));
#else
      Hasher local;
      Hasher& snap = scratch ? *scratch : local;
      snap.snapshot_from(h);
      snap.update("zig-stark:sample", 16);
      uint8_t cb[8];
      for (int i = 0; i < 8; ++i) cb[i] = (uint8_t)(counter >> (8 * i));
      snap.update(cb, 8);
      snap.finalize(blk);
#endif
      h.update(blk, 32);
      const size_t k = len < 32 ? len : 32;
      copy_bytes(out, blk, k);
      out += k;
      len -= k;
      ++counter;
    }
  }
  ZS_HD qm31 sample_q(Hasher* scratch = nullptr) {
    uint8_t b[16];
    sample_bytes(b, 16, scratch);
    return qmake(m31_from_le(b), m31_from_le(b + 4), m31_from_le(b + 8), m31_from_le(b + 12));
  }
  // channel.zig:79-101.
  uint64_t sample_index(uint64_t n) {
    unsigned lg = 0;
    while ((n >> (lg + 1)) != 0) ++lg;
    const unsigned bits = lg + 1, nbytes = (bits + 7) / 8;
    const uint64_t mask = bits >= 64 ? ~0ull : (((uint64_t)1 << bits) - 1);
    for (;;) {
      uint8_t buf[8];
      sample_bytes(buf, nbytes);
      uint64_t v = 0;
      for (unsigned i = 0; i < nbytes; ++i) v = (v << 8) | buf[i];
      v &= mask;
      if (v < n) return v;
    }
  }
};

#ifdef __CUDACC__
// Block-cooperative copy of a transcript state between global and shared memory (the
// single-thread transcript steps run on the shared copy: byte-wise state updates cost
// far less there than in global memory).
__device__ __forceinline__ void copy_state(void* dst, const void* src, size_t bytes) {
  uint2* d = static_cast<uint2*>(dst);
  const uint2* s = static_cast<const uint2*>(src);
  for (size_t i = threadIdx.x; i < bytes / 8; i += blockDim.x) d[i] = s[i];
}
static_assert(sizeof(Channel) % 8 == 0, "the transcript state is copied in 8-byte words");
#endif

// Lagrange interpolation through (xs[i], ys[i]), the reference's own O(n^2)
// algorithm (univariate.zig:79-139); used on <= 8 points (AIR constants, the FRI
// remainder).
inline std::vector<qm31> interpolate_small(const std::vector<qm31>& xs, const std::vector<qm31>& ys) {
  const size_t n = xs.size();
  std::vector<qm31> p(n + 1, qzero());
  p[0] = qone();
  size_t plen = 1;
  for (const qm31& xi : xs) {
    for (size_t j = plen; j > 0; --j) p[j] = qsub(p[j - 1], qmul(p[j], xi));
    p[0] = qmul(qneg(p[0]), xi);
    ++plen;
  }
  std::vector<qm31> acc(n, qzero()), tmp(n);
  for (size_t i = 0; i < n; ++i) {
    qm31 w = qone();
    for (size_t j = 0; j < n; ++j)
      if (i != j) w = qmul(w, qsub(xs[i], xs[j]));
    const qm31 scale = qmul(ys[i], qinv(w));
    tmp[n - 1] = p[n];
    for (size_t j = n - 1; j > 0; --j) tmp[j - 1] = qadd(p[j], qmul(xs[i], tmp[j]));
    for (size_t k = 0; k < n; ++k) acc[k] = qadd(acc[k], qmul(tmp[k], scale));
  }
  return acc;
}

}  // namespace zs
