// ORACLE — test infrastructure only. A CPU restatement of the reference's field
// tower, used as the checker for the GPU backend. Nothing in the product links it.
//
// M31  = F_(2^31-1)                      src/m31/field/m31.zig
// CM31 = M31[i] / (i^2 + 1)              src/m31/field/cm31.zig
// QM31 = CM31[j] / (j^2 + i)             src/m31/field/qm31.zig
//
// Every operation returns the canonical representative in [0, p), exactly like
// the reference, so any algebraically equal computation gives identical bytes.
#pragma once
#include <cstdint>
#include <cstring>

namespace orc {

constexpr uint32_t P = 2147483647u;  // m31.zig:10
constexpr uint64_t P64 = 2147483647ull;

struct M31 {
  uint32_t v = 0;
  M31() = default;
  explicit constexpr M31(uint32_t x) : v(x) {}

  // m31.zig:19-22 fromInt: reduce x mod p when x >= p.
  static M31 fromInt(uint32_t x) { return M31(x >= P ? x % P : x); }
  static M31 fromInt64(uint64_t x) { return M31((uint32_t)(x % P64)); }
  static M31 zero() { return M31(0); }
  static M31 one() { return M31(1); }

  // m31.zig:28-35 add: 64-bit sum, subtract p once, Mersenne fold, subtract once.
  M31 add(M31 o) const {
    uint64_t r = (uint64_t)v + (uint64_t)o.v;
    if (r >= P64) r -= P64;
    r = (r & P64) + (r >> 31);
    if (r >= P64) r -= P64;
    return M31((uint32_t)r);
  }
  // m31.zig:37-42 sub.
  M31 sub(M31 o) const {
    if (v >= o.v) return M31(v - o.v);
    return M31(P - (o.v - v));
  }
  // m31.zig:44-52 mul: 32x32->64 product, lo = prod & p, hi = prod >> 31,
  // sum and two conditional subtractions.
  M31 mul(M31 o) const {
    uint64_t prod = (uint64_t)v * (uint64_t)o.v;
    uint32_t lo = (uint32_t)(prod & P64);
    uint32_t hi = (uint32_t)(prod >> 31);
    uint64_t r = (uint64_t)lo + (uint64_t)hi;
    if (r >= P64) r -= P64;
    if (r >= P64) r -= P64;
    return M31((uint32_t)r);
  }
  // m31.zig:54-57 neg.
  M31 neg() const { return v == 0 ? *this : M31(P - v); }
  // m31.zig:64-73 pow (square and multiply on a u32 exponent).
  M31 pow(uint32_t e) const {
    M31 r = one(), b = *this;
    while (e > 0) {
      if (e & 1) r = r.mul(b);
      b = b.mul(b);
      e >>= 1;
    }
    return r;
  }
  // m31.zig:59-62 inv = x^(p-2). The reference asserts x != 0 only in debug
  // builds; in release 0^(p-2) = 0, which is what this returns for 0.
  M31 inv() const { return pow(P - 2); }
  bool eq(M31 o) const { return v == o.v; }
  // m31.zig:93-100 little-endian 4 bytes; fromBytes reduces raw % p.
  void toBytes(uint8_t* out) const { std::memcpy(out, &v, 4); }
  static M31 fromBytes(const uint8_t* b) {
    uint32_t raw;
    std::memcpy(&raw, b, 4);
    return fromInt(raw);
  }
};

struct CM31 {
  M31 c0, c1;
  CM31() = default;
  CM31(M31 a, M31 b) : c0(a), c1(b) {}
  static CM31 fromM31(M31 x) { return CM31(x, M31::zero()); }
  static CM31 zero() { return CM31(M31::zero(), M31::zero()); }
  static CM31 one() { return CM31(M31::one(), M31::zero()); }
  static CM31 i() { return CM31(M31::zero(), M31::one()); }
  CM31 add(CM31 o) const { return CM31(c0.add(o.c0), c1.add(o.c1)); }  // cm31.zig:16-21
  CM31 sub(CM31 o) const { return CM31(c0.sub(o.c0), c1.sub(o.c1)); }  // cm31.zig:23-28
  // cm31.zig:30-39 schoolbook product with i^2 = -1.
  CM31 mul(CM31 o) const {
    M31 ac = c0.mul(o.c0), bd = c1.mul(o.c1), ad = c0.mul(o.c1), bc = c1.mul(o.c0);
    return CM31(ac.sub(bd), ad.add(bc));
  }
  CM31 neg() const { return CM31(c0.neg(), c1.neg()); }  // cm31.zig:41-43
  // cm31.zig:45-52 inverse through the norm c0^2 + c1^2.
  CM31 inv() const {
    M31 norm = c0.mul(c0).add(c1.mul(c1));
    M31 ni = norm.inv();
    return CM31(c0.mul(ni), c1.neg().mul(ni));
  }
  CM31 mulByI() const { return CM31(c1.neg(), c0); }  // cm31.zig:68-70
  bool eq(CM31 o) const { return c0.eq(o.c0) && c1.eq(o.c1); }
  void toBytes(uint8_t* out) const { c0.toBytes(out); c1.toBytes(out + 4); }  // cm31.zig:74-84
  static CM31 fromBytes(const uint8_t* b) { return CM31(M31::fromBytes(b), M31::fromBytes(b + 4)); }
};

struct QM31 {
  CM31 a, b;
  QM31() = default;
  QM31(CM31 x, CM31 y) : a(x), b(y) {}
  static QM31 fromM31(M31 x) { return QM31(CM31::fromM31(x), CM31::zero()); }
  static QM31 fromU32(uint32_t x) { return fromM31(M31::fromInt(x)); }
  static QM31 make(uint32_t a0, uint32_t a1, uint32_t b0, uint32_t b1) {
    return QM31(CM31(M31(a0), M31(a1)), CM31(M31(b0), M31(b1)));
  }
  static QM31 zero() { return QM31(CM31::zero(), CM31::zero()); }
  static QM31 one() { return QM31(CM31::one(), CM31::zero()); }
  QM31 add(QM31 o) const { return QM31(a.add(o.a), b.add(o.b)); }  // qm31.zig:17-19
  QM31 sub(QM31 o) const { return QM31(a.sub(o.a), b.sub(o.b)); }  // qm31.zig:21-23
  // qm31.zig:25-33: ab0 = a*a', ab1 = b*b', cross = (a+b)(a'+b');
  // result = (ab0 - i*ab1, cross - ab0 - ab1)  (j^2 = -i).
  QM31 mul(QM31 o) const {
    CM31 ab0 = a.mul(o.a), ab1 = b.mul(o.b);
    CM31 cross = a.add(b).mul(o.a.add(o.b));
    return QM31(ab0.sub(ab1.mulByI()), cross.sub(ab0).sub(ab1));
  }
  QM31 neg() const { return QM31(a.neg(), b.neg()); }
  // qm31.zig:39-48 inverse through the CM31 norm a^2 + i*b^2.
  QM31 inv() const {
    CM31 a2 = a.mul(a);
    CM31 b2i = b.mul(b).mulByI();
    CM31 ni = a2.add(b2i).inv();
    return QM31(a.mul(ni), b.neg().mul(ni));
  }
  // qm31.zig:57-67 square and multiply on a u64 exponent.
  QM31 pow(uint64_t e) const {
    QM31 base = *this, r = one();
    while (e > 0) {
      if (e & 1) r = r.mul(base);
      base = base.mul(base);
      e >>= 1;
    }
    return r;
  }
  bool eq(QM31 o) const { return a.eq(o.a) && b.eq(o.b); }
  bool isZero() const { return a.c0.v == 0 && a.c1.v == 0 && b.c0.v == 0 && b.c1.v == 0; }
  // qm31.zig:91-101: a.c0 | a.c1 | b.c0 | b.c1, each u32 LE.
  void toBytes(uint8_t* out) const { a.toBytes(out); b.toBytes(out + 8); }
  static QM31 fromBytes(const uint8_t* x) { return QM31(CM31::fromBytes(x), CM31::fromBytes(x + 8)); }

  // qm31.zig:80-83 TWO_ADIC_ROOT: a primitive 2^32-th root of unity.
  static QM31 twoAdicRoot() {
    static const uint8_t bytes[16] = {0x60, 0x1f, 0x3d, 0x34, 0x32, 0x39, 0xa0, 0x6a,
                                      0xa0, 0xd6, 0x51, 0x61, 0x91, 0xe7, 0x86, 0x3e};
    return fromBytes(bytes);
  }
  // qm31.zig:86-89 primitiveRootOfUnity(log) = R^(2^(32-log)).
  static QM31 primitiveRootOfUnity(unsigned log_size) {
    return twoAdicRoot().pow((uint64_t)1 << (32 - log_size));
  }
};

// fri.zig:36 FRI_OFFSET = 1 + i.
inline QM31 friOffset() { return QM31(CM31::one(), CM31::one()); }

}  // namespace orc
