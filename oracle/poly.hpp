// ORACLE — test infrastructure only. Univariate QM31 polynomials.
//   src/m31/poly/univariate.zig  eval (Horner) 11-19, interpolate (O(n^2)) 79-139
//
// `evalHorner` and `interpolateLagrange` are the faithful restatements. The
// radix-2 NTT helpers compute the same unique polynomial / the same
// evaluations (QM31 is the ring CM31[j]/(j^2+i); both of its CM31 components
// see the 2-adic root with order exactly 2^32, so every difference of two
// distinct points of a 2-power subgroup is a unit and interpolation on it is
// unique). The tests assert byte equality of both routes before the NTT route
// is trusted at sizes where O(n^2) is out of reach.
#pragma once
#include <vector>

#include "field.hpp"

namespace orc {

// univariate.zig:11-19.
inline QM31 evalHorner(const std::vector<QM31>& poly, const QM31& x) {
  QM31 r = QM31::zero();
  for (size_t i = poly.size(); i > 0; --i) r = r.mul(x).add(poly[i - 1]);
  return r;
}

// univariate.zig:79-139, step for step.
inline std::vector<QM31> interpolateLagrange(const std::vector<QM31>& xs,
                                             const std::vector<QM31>& ys) {
  size_t n = xs.size();
  // P(z) = prod (z - x_i), length n+1 (univariate.zig:89-103)
  std::vector<QM31> p(n + 1, QM31::zero());
  p[0] = QM31::one();
  size_t plen = 1;
  for (const QM31& xi : xs) {
    for (size_t j = plen; j > 0; --j) p[j] = p[j - 1].sub(p[j].mul(xi));
    p[0] = p[0].neg().mul(xi);
    ++plen;
  }
  // weights w_i = prod_{j != i} (x_i - x_j) (univariate.zig:105-114)
  std::vector<QM31> weights(n);
  for (size_t i = 0; i < n; ++i) {
    QM31 w = QM31::one();
    for (size_t j = 0; j < n; ++j)
      if (i != j) w = w.mul(xs[i].sub(xs[j]));
    weights[i] = w;
  }
  // sum_i y_i / w_i * P(z)/(z - x_i) (univariate.zig:116-136)
  std::vector<QM31> acc(n, QM31::zero()), tmp2(n);
  for (size_t i = 0; i < n; ++i) {
    QM31 scale = ys[i].mul(weights[i].inv());
    tmp2[n - 1] = p[n];
    for (size_t j = n - 1; j > 0; --j) tmp2[j - 1] = p[j].add(xs[i].mul(tmp2[j]));
    for (size_t k = 0; k < n; ++k) acc[k] = acc[k].add(tmp2[k].mul(scale));
  }
  return acc;
}

inline unsigned log2Exact(size_t n) {
  unsigned l = 0;
  while (((size_t)1 << l) < n) ++l;
  return l;
}

// In-place radix-2 DFT: a[i] <- sum_k a[k] * root^(i k), size a power of two.
inline void nttInPlace(std::vector<QM31>& a, const QM31& root) {
  size_t n = a.size();
  if (n <= 1) return;
  unsigned lg = log2Exact(n);
  for (size_t i = 0; i < n; ++i) {
    size_t r = 0;
    for (unsigned b = 0; b < lg; ++b) r |= ((i >> b) & 1) << (lg - 1 - b);
    if (i < r) std::swap(a[i], a[r]);
  }
  for (size_t len = 2; len <= n; len <<= 1) {
    QM31 wl = root.pow(n / len);
    std::vector<QM31> tw(len / 2);
    tw[0] = QM31::one();
    for (size_t k = 1; k < len / 2; ++k) tw[k] = tw[k - 1].mul(wl);
    for (size_t s = 0; s < n; s += len)
      for (size_t k = 0; k < len / 2; ++k) {
        QM31 u = a[s + k], v = a[s + k + len / 2].mul(tw[k]);
        a[s + k] = u.add(v);
        a[s + k + len / 2] = u.sub(v);
      }
  }
}

// Coefficients of the degree < n polynomial through (w^i, ys[i]), w of order n.
inline std::vector<QM31> interpolateSubgroupNtt(const std::vector<QM31>& ys, unsigned log_n) {
  std::vector<QM31> c = ys;
  QM31 w = QM31::primitiveRootOfUnity(log_n);
  nttInPlace(c, w.inv());
  QM31 ninv = QM31::fromU32((uint32_t)c.size()).inv();
  for (auto& v : c) v = v.mul(ninv);
  return c;
}

// Evaluations of `coeffs` on offset * <w_N>, natural order, N = 2^log_N.
inline std::vector<QM31> evaluateCosetNtt(const std::vector<QM31>& coeffs, const QM31& offset,
                                          unsigned log_N) {
  size_t N = (size_t)1 << log_N;
  std::vector<QM31> a(N, QM31::zero());
  QM31 s = QM31::one();
  for (size_t k = 0; k < coeffs.size(); ++k) {
    a[k] = coeffs[k].mul(s);
    s = s.mul(offset);
  }
  nttInPlace(a, QM31::primitiveRootOfUnity(log_N));
  return a;
}

}  // namespace orc
