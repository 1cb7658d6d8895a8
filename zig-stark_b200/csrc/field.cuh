// Exact M31 / CM31 / QM31 arithmetic for host and device.
//
// Field tower of the reference: M31 = F_(2^31-1) (src/m31/field/m31.zig),
// CM31 = M31[i]/(i^2+1) (cm31.zig), QM31 = CM31[j]/(j^2+i) (qm31.zig).
// Every function returns the canonical representative in [0, p), the same value
// the reference computes, so results are bit-identical to it whatever the
// evaluation order (the tower is a commutative ring and all operations are exact).
//
// Reductions use one conditional subtraction expressed as an unsigned min:
//   add: a + b < 2p        -> min(s, s - p)
//   sub: a - b (mod 2^32)  -> min(d, d + p)
//   mul: (a*b & p) + (a*b >> 31) <= 2p - 3 for a, b < p -> min(s, s - p)
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define ZS_HD __host__ __device__ __forceinline__
#else
#define ZS_HD inline
#endif

namespace zs {

constexpr uint32_t P = 2147483647u;

ZS_HD uint32_t umin32(uint32_t a, uint32_t b) { return a < b ? a : b; }

ZS_HD uint32_t madd(uint32_t a, uint32_t b) {
  uint32_t s = a + b;
  return umin32(s, s - P);
}
ZS_HD uint32_t msub(uint32_t a, uint32_t b) {
  uint32_t d = a - b;
  return umin32(d, d + P);
}
ZS_HD uint32_t mneg(uint32_t a) { return a == 0 ? 0 : P - a; }
ZS_HD uint32_t mmul(uint32_t a, uint32_t b) {
  uint64_t prod = (uint64_t)a * (uint64_t)b;
  uint32_t s = ((uint32_t)prod & P) + (uint32_t)(prod >> 31);
  return umin32(s, s - P);
}
// x * 2^k mod p for 0 <= k < 31: a rotation inside the 31-bit word.
ZS_HD uint32_t mshl(uint32_t x, unsigned k) {
  uint32_t r = ((x << k) | (x >> (31 - k))) & P;
  return r == P ? 0 : r;
}
ZS_HD uint32_t mpow(uint32_t a, uint32_t e) {
  uint32_t r = 1;
  while (e) {
    if (e & 1) r = mmul(r, a);
    a = mmul(a, a);
    e >>= 1;
  }
  return r;
}
// a^(p-2); 0 maps to 0 exactly as the reference's release build does.
ZS_HD uint32_t minv(uint32_t a) { return mpow(a, P - 2); }

struct cm31 {
  uint32_t a, b;  // a + b i
};
ZS_HD cm31 cadd(cm31 x, cm31 y) { return {madd(x.a, y.a), madd(x.b, y.b)}; }
ZS_HD cm31 csub(cm31 x, cm31 y) { return {msub(x.a, y.a), msub(x.b, y.b)}; }
ZS_HD cm31 cneg(cm31 x) { return {mneg(x.a), mneg(x.b)}; }
// Karatsuba: (a+bi)(c+di) = (ac - bd) + ((a+b)(c+d) - ac - bd) i.
ZS_HD cm31 cmul(cm31 x, cm31 y) {
  uint32_t ac = mmul(x.a, y.a), bd = mmul(x.b, y.b);
  uint32_t t = mmul(madd(x.a, x.b), madd(y.a, y.b));
  return {msub(ac, bd), msub(msub(t, ac), bd)};
}
ZS_HD cm31 cmul_m(cm31 x, uint32_t s) { return {mmul(x.a, s), mmul(x.b, s)}; }
ZS_HD cm31 cmul_i(cm31 x) { return {mneg(x.b), x.a}; }
// (a+bi)^-1 = (a - bi) / (a^2 + b^2); a zero norm gives zero like the reference.
ZS_HD cm31 cinv(cm31 x) {
  uint32_t ni = minv(madd(mmul(x.a, x.a), mmul(x.b, x.b)));
  return {mmul(x.a, ni), mmul(mneg(x.b), ni)};
}

struct qm31 {
  cm31 a, b;  // a + b j, j^2 = -i. Wire order: a.a, a.b, b.a, b.b (qm31.zig:91-94)
};
ZS_HD qm31 qzero() { return {{0, 0}, {0, 0}}; }
ZS_HD qm31 qone() { return {{1, 0}, {0, 0}}; }
ZS_HD qm31 qfrom_m31(uint32_t v) { return {{v, 0}, {0, 0}}; }
ZS_HD qm31 qmake(uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3) { return {{w0, w1}, {w2, w3}}; }
ZS_HD qm31 qadd(qm31 x, qm31 y) { return {cadd(x.a, y.a), cadd(x.b, y.b)}; }
ZS_HD qm31 qsub(qm31 x, qm31 y) { return {csub(x.a, y.a), csub(x.b, y.b)}; }
ZS_HD qm31 qneg(qm31 x) { return {cneg(x.a), cneg(x.b)}; }
// qm31.zig:25-33 structure: (ab0 - i ab1, (a+b)(a'+b') - ab0 - ab1).
ZS_HD qm31 qmul(qm31 x, qm31 y) {
  cm31 ab0 = cmul(x.a, y.a), ab1 = cmul(x.b, y.b);
  cm31 cross = cmul(cadd(x.a, x.b), cadd(y.a, y.b));
  return {csub(ab0, cmul_i(ab1)), csub(csub(cross, ab0), ab1)};
}
ZS_HD qm31 qmul_m(qm31 x, uint32_t s) { return {cmul_m(x.a, s), cmul_m(x.b, s)}; }
ZS_HD qm31 qmul_c(qm31 x, cm31 s) { return {cmul(x.a, s), cmul(x.b, s)}; }
// Norm a^2 + i b^2 in CM31; inverse = (a - b j) / norm (qm31.zig:39-48).
ZS_HD cm31 qnorm(qm31 x) { return cadd(cmul(x.a, x.a), cmul_i(cmul(x.b, x.b))); }
ZS_HD qm31 qinv(qm31 x) {
  cm31 ni = cinv(qnorm(x));
  return {cmul(x.a, ni), cmul(cneg(x.b), ni)};
}
ZS_HD qm31 qpow(qm31 x, uint64_t e) {
  qm31 r = qone();
  while (e) {
    if (e & 1) r = qmul(r, x);
    x = qmul(x, x);
    e >>= 1;
  }
  return r;
}
ZS_HD bool qeq(qm31 x, qm31 y) { return x.a.a == y.a.a && x.a.b == y.a.b && x.b.a == y.b.a && x.b.b == y.b.b; }

// qm31.zig:80-83: the primitive 2^32-th root of unity, as LE words.
ZS_HD qm31 q_two_adic_root() { return qmake(0x343d1f60u, 0x6aa03932u, 0x6151d6a0u, 0x3e86e791u); }
ZS_HD qm31 q_root_of_unity(unsigned log_size) {
  return qpow(q_two_adic_root(), (uint64_t)1 << (32 - log_size));
}
// fri.zig:36: FRI_OFFSET = {a = CM31 one, b = CM31 one} = 1 + j.
ZS_HD qm31 q_fri_offset() { return qmake(1, 0, 1, 0); }

// Circle group point over M31 (src/m31/circle/point.zig).
struct cpoint {
  uint32_t x, y;
};
ZS_HD cpoint padd(cpoint p, cpoint q) {
  return {msub(mmul(p.x, q.x), mmul(p.y, q.y)), madd(mmul(p.x, q.y), mmul(p.y, q.x))};
}
ZS_HD cpoint pdbl(cpoint p) { return {msub(mmul(p.x, p.x), mmul(p.y, p.y)), mmul(mmul(p.x, p.y), 2)}; }
ZS_HD cpoint pneg(cpoint p) { return {p.x, mneg(p.y)}; }
ZS_HD cpoint pmul(cpoint p, uint64_t k) {
  cpoint r = {1, 0};
  while (k) {
    if (k & 1) r = padd(r, p);
    p = pdbl(p);
    k >>= 1;
  }
  return r;
}

}  // namespace zs
