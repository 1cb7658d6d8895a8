// ORACLE — test infrastructure only. Circle group, cosets and the circle FFT
// over M31, restated from:
//   src/m31/circle/point.zig  add 16-21, double 23-28, generator 49-51,
//                             mulScalar 64-86
//   src/m31/circle/coset.zig  at 23-26, half 38-41, conjugate 44-46,
//                             canonicHalf 59-65
//   src/m31/ntt/circle.zig    butterfly 27-37, fftLayerLoop 39-55,
//                             slowPrecomputeTwiddles 69-82, lineTwiddleSlice 86-91,
//                             circleTwiddles 96-106, circleFFT 195-246,
//                             evalAtPoint 250-258, circleIFFT 272-346
#pragma once
#include <cstdint>
#include <vector>

#include "field.hpp"

namespace orc {

struct CirclePoint {
  M31 x, y;
  CirclePoint() = default;
  CirclePoint(M31 a, M31 b) : x(a), y(b) {}
  static CirclePoint identity() { return CirclePoint(M31::one(), M31::zero()); }
  static CirclePoint generator() { return CirclePoint(M31(1268011823u), M31(2u)); }
  CirclePoint add(const CirclePoint& o) const {
    return CirclePoint(x.mul(o.x).sub(y.mul(o.y)), x.mul(o.y).add(y.mul(o.x)));
  }
  CirclePoint dbl() const {
    return CirclePoint(x.mul(x).sub(y.mul(y)), x.mul(y).mul(M31(2)));
  }
  CirclePoint neg() const { return CirclePoint(x, y.neg()); }
  bool isIdentity() const { return x.v == 1 && y.v == 0; }
  // point.zig:64-86: fixed window of width 4 over all 64 scalar bits.
  CirclePoint mulScalar(uint64_t scalar) const {
    CirclePoint table[16];
    table[0] = identity();
    table[1] = *this;
    table[2] = add(*this);
    for (int i = 3; i < 16; ++i) table[i] = table[i - 1].add(*this);
    CirclePoint r = identity();
    for (int d = 15; d >= 0; --d) {
      r = r.dbl().dbl().dbl().dbl();
      r = r.add(table[(scalar >> (4 * d)) & 0xf]);
    }
    return r;
  }
};

struct CircleCoset {
  CirclePoint offset, step;
  unsigned log_size;
  CircleCoset(CirclePoint o, CirclePoint s, unsigned l) : offset(o), step(s), log_size(l) {}
  size_t size() const { return (size_t)1 << log_size; }
  CirclePoint at(size_t i) const { return offset.add(step.mulScalar(i)); }
  CircleCoset half() const { return CircleCoset(offset.dbl(), step.dbl(), log_size - 1); }
  CircleCoset conjugate() const { return CircleCoset(offset.neg(), step.neg(), log_size); }
  // coset.zig:59-65 (log_size of the full domain; returns the half coset).
  static CircleCoset canonicHalf(unsigned log_size) {
    CirclePoint gen = CirclePoint::generator().neg();
    CirclePoint off = gen.mulScalar((uint64_t)1 << (30 - log_size));
    CirclePoint st = gen.mulScalar((uint64_t)1 << (32 - log_size));
    return CircleCoset(off, st, log_size - 1);
  }
};

inline void bitReverseM31(std::vector<M31>& v, size_t off, size_t len) {
  unsigned width = 0;
  while (((size_t)1 << width) < len) ++width;
  for (size_t i = 0; i < len; ++i) {
    size_t r = 0, x = i;
    for (unsigned b = 0; b < width; ++b) {
      r = (r << 1) | (x & 1);
      x >>= 1;
    }
    if (i < r) std::swap(v[off + i], v[off + r]);
  }
}

// circle.zig:69-82. `cache_points` selects the per-point `at()` evaluation of the
// reference (true) or an incremental walk along the coset (false, same values).
inline std::vector<M31> precomputeTwiddles(const CircleCoset& half_coset, bool faithful = true) {
  std::vector<M31> out(half_coset.size());
  size_t pos = 0;
  CircleCoset cur = half_coset;
  for (unsigned k = half_coset.log_size; k > 0; --k) {
    size_t m = (size_t)1 << (k - 1);
    if (faithful) {
      for (size_t i = 0; i < m; ++i) out[pos + i] = cur.at(i).x;
    } else {
      CirclePoint pt = cur.offset;
      for (size_t i = 0; i < m; ++i) {
        out[pos + i] = pt.x;
        pt = pt.add(cur.step);
      }
    }
    bitReverseM31(out, pos, m);
    pos += m;
    cur = cur.half();
  }
  out[pos] = M31::one();
  return out;
}

// circle.zig:86-91: offset of the j-th line twiddle layer (0 = largest).
inline size_t lineTwiddleOffset(size_t blen, unsigned j, unsigned lg) {
  size_t len = (size_t)1 << (lg - 2 - j);
  return blen - 2 * len;
}
inline size_t lineTwiddleLen(unsigned j, unsigned lg) { return (size_t)1 << (lg - 2 - j); }

// circle.zig:96-106: [y, -y, -x, x] per (x, y) pair of the first line layer.
inline std::vector<M31> circleTwiddles(const M31* first, size_t len) {
  std::vector<M31> out(2 * len);
  for (size_t i = 0; i < len / 2; ++i) {
    M31 x = first[2 * i], y = first[2 * i + 1];
    out[4 * i] = y;
    out[4 * i + 1] = y.neg();
    out[4 * i + 2] = x.neg();
    out[4 * i + 3] = x;
  }
  return out;
}

// circle.zig:39-55 with butterfly/ibutterfly (27-37).
inline void fftLayerLoop(std::vector<M31>& v, unsigned i, size_t h, M31 t, bool inverse) {
  size_t step = (size_t)1 << i;
  size_t base = h << (i + 1);
  for (size_t l = 0; l < step; ++l) {
    size_t i0 = base + l, i1 = i0 + step;
    M31 v0 = v[i0], v1 = v[i1];
    if (inverse) {
      M31 tmp = v0;
      v0 = tmp.add(v1);
      v1 = tmp.sub(v1).mul(t);
    } else {
      M31 tmp = v1.mul(t);
      v1 = v0.sub(tmp);
      v0 = v0.add(tmp);
    }
    v[i0] = v0;
    v[i1] = v1;
  }
}

// circle.zig:195-246. `tw` may pass precomputed twiddles for `half_coset`.
inline std::vector<M31> circleFFT(const std::vector<M31>& coeffs, const CircleCoset& half_coset,
                                  const std::vector<M31>* tw = nullptr, bool faithful = true) {
  size_t n = coeffs.size(), half = n / 2;
  unsigned lg = 0;
  while (((size_t)1 << lg) < n) ++lg;
  std::vector<M31> ev(n);
  for (size_t i = 0; i < half; ++i) {
    ev[2 * i] = coeffs[i];
    ev[2 * i + 1] = coeffs[half + i];
  }
  auto bf = [&](size_t a, size_t b, M31 t) {
    M31 tmp = ev[b].mul(t);
    ev[b] = ev[a].sub(tmp);
    ev[a] = ev[a].add(tmp);
  };
  if (lg == 1) {
    bf(0, 1, half_coset.at(0).y);
  } else if (lg == 2) {
    CirclePoint p = half_coset.at(0);
    bf(0, 2, p.x);
    bf(1, 3, p.x);
    bf(0, 1, p.y);
    bf(2, 3, p.y.neg());
  } else {
    std::vector<M31> local;
    if (!tw) {
      local = precomputeTwiddles(half_coset, faithful);
      tw = &local;
    }
    for (unsigned jj = 0; jj < lg - 1; ++jj) {
      unsigned j = (lg - 2) - jj;
      size_t off = lineTwiddleOffset(half, j, lg), len = lineTwiddleLen(j, lg);
      for (size_t h = 0; h < len; ++h) fftLayerLoop(ev, j + 1, h, (*tw)[off + h], false);
    }
    std::vector<M31> ct = circleTwiddles(tw->data() + lineTwiddleOffset(half, 0, lg), lineTwiddleLen(0, lg));
    for (size_t h = 0; h < ct.size(); ++h) fftLayerLoop(ev, 0, h, ct[h], false);
  }
  bitReverseM31(ev, 0, n);
  return ev;
}

// circle.zig:272-346. `tw` may pass precomputed (non-inverted) twiddles.
inline std::vector<M31> circleIFFT(const std::vector<M31>& evals, const CircleCoset& half_coset,
                                   const std::vector<M31>* tw = nullptr, bool faithful = true) {
  size_t n = evals.size(), half = n / 2;
  unsigned lg = 0;
  while (((size_t)1 << lg) < n) ++lg;
  std::vector<M31> v = evals;
  bitReverseM31(v, 0, n);
  auto ibf = [&](size_t a, size_t b, M31 t) {
    M31 tmp = v[a];
    v[a] = tmp.add(v[b]);
    v[b] = tmp.sub(v[b]).mul(t);
  };
  if (lg == 1) {
    M31 y = half_coset.at(0).y;
    M31 yn_inv = y.mul(M31(2)).inv();
    M31 y_inv = yn_inv.mul(M31(2));
    M31 n_inv = yn_inv.mul(y);
    ibf(0, 1, y_inv);
    v[0] = v[0].mul(n_inv);
    v[1] = v[1].mul(n_inv);
  } else if (lg == 2) {
    CirclePoint p = half_coset.at(0);
    M31 x = p.x, y = p.y;
    M31 xyn_inv = x.mul(y).mul(M31(4)).inv();
    M31 x_inv = xyn_inv.mul(y).mul(M31(4));
    M31 y_inv = xyn_inv.mul(x).mul(M31(4));
    M31 n_inv = xyn_inv.mul(x).mul(y);
    ibf(0, 1, y_inv);
    ibf(2, 3, y_inv.neg());
    ibf(0, 2, x_inv);
    ibf(1, 3, x_inv);
    for (int k = 0; k < 4; ++k) v[k] = v[k].mul(n_inv);
  } else {
    std::vector<M31> t = tw ? *tw : precomputeTwiddles(half_coset, faithful);
    for (auto& x : t) x = x.inv();
    std::vector<M31> ct = circleTwiddles(t.data() + lineTwiddleOffset(half, 0, lg), lineTwiddleLen(0, lg));
    for (size_t h = 0; h < ct.size(); ++h) fftLayerLoop(v, 0, h, ct[h], true);
    for (unsigned j = 0; j < lg - 1; ++j) {
      size_t off = lineTwiddleOffset(half, j, lg), len = lineTwiddleLen(j, lg);
      for (size_t h = 0; h < len; ++h) fftLayerLoop(v, j + 1, h, t[off + h], true);
    }
    M31 inv_n = M31::fromInt((uint32_t)n).inv();
    for (auto& x : v) x = x.mul(inv_n);
  }
  std::vector<M31> coeffs(n);
  for (size_t i = 0; i < half; ++i) {
    coeffs[i] = v[2 * i];
    coeffs[half + i] = v[2 * i + 1];
  }
  return coeffs;
}

// circle.zig:108-127, 169-183, 250-258: the O(n) fold evaluation at one point.
inline M31 circlePi(M31 x) { return x.mul(x).mul(M31(2)).sub(M31::one()); }
inline M31 foldRange(const std::vector<M31>& c, size_t half, size_t start, size_t len,
                     const M31* facs) {
  if (len == 1) {
    size_t k = start;
    return (k % 2 == 0) ? c[k / 2] : c[half + (k - 1) / 2];
  }
  size_t h = len / 2;
  M31 lhs = foldRange(c, half, start, h, facs + 1);
  M31 rhs = foldRange(c, half, start + h, h, facs + 1);
  return lhs.add(rhs.mul(facs[0]));
}
inline M31 circleEvalAtPoint(const std::vector<M31>& coeffs, const CirclePoint& pt) {
  size_t n = coeffs.size();
  if (n == 1) return coeffs[0];
  unsigned lg = 0;
  while (((size_t)1 << lg) < n) ++lg;
  M31 al[32];
  al[lg - 1] = pt.y;
  M31 x = pt.x;
  for (size_t i = lg - 1; i > 0;) {
    --i;
    al[i] = x;
    x = circlePi(x);
  }
  return foldRange(coeffs, n / 2, 0, n, al);
}
inline CirclePoint circleDomainPoint(const CircleCoset& half_coset, size_t i) {
  size_t h = half_coset.size();
  return i < h ? half_coset.at(i) : half_coset.conjugate().at(i - h);
}

}  // namespace orc
