// ORACLE — test infrastructure only. FRI over QM31, restated from
// src/m31/fri.zig: domainPoint 96-101, domainPoints 104-117, foldValue 125-130,
// proveCodeword 157-273, verify 277-336.
#pragma once
#include <vector>

#include "hash.hpp"
#include "poly.hpp"
#include "wire.hpp"

namespace orc {

inline QM31 invTwo() { return QM31::fromM31(M31(2).inv()); }

// fri.zig:96-101.
inline QM31 friDomainPoint(const FriParams& p, unsigned layer, size_t j) {
  unsigned dlog = p.domainLogSize();
  QM31 w = QM31::primitiveRootOfUnity(dlog - layer);
  QM31 off = friOffset().pow((uint64_t)1 << layer);
  return off.mul(w.pow(j));
}

// fri.zig:104-117.
inline std::vector<QM31> friDomainPoints(const FriParams& p, unsigned layer) {
  unsigned dlog = p.domainLogSize();
  size_t n = (size_t)1 << (dlog - layer);
  std::vector<QM31> pts(n);
  QM31 w = QM31::primitiveRootOfUnity(dlog - layer);
  QM31 acc = friOffset().pow((uint64_t)1 << layer);
  for (size_t j = 0; j < n; ++j) {
    pts[j] = acc;
    acc = acc.mul(w);
  }
  return pts;
}

// fri.zig:125-130.
inline QM31 friFoldValue(const QM31& g, const QM31& y0, const QM31& y1, const QM31& alpha) {
  QM31 it = invTwo();
  QM31 half_sum = y0.add(y1).mul(it);
  QM31 half_diff = y0.sub(y1).mul(g.inv()).mul(it);
  return half_sum.add(alpha.mul(half_diff));
}

inline std::vector<Digest> hashCodeword(const std::vector<QM31>& cw) {
  std::vector<Digest> leaves(cw.size());
  for (size_t i = 0; i < cw.size(); ++i) leaves[i] = hashQM31(cw[i]);
  return leaves;
}

// fri.zig:157-273. `layers_out`, when given, receives every layer (0..L).
inline FriProof friProveCodeword(const FriParams& params, const std::vector<QM31>& codeword,
                                 Channel& ch, std::vector<std::vector<QM31>>* layers_out = nullptr) {
  unsigned L = params.numFoldRounds();
  unsigned dlog = params.domainLogSize();
  size_t n0 = (size_t)1 << dlog;
  std::vector<std::vector<QM31>> doms(L + 1);
  for (unsigned i = 0; i <= L; ++i) doms[i] = friDomainPoints(params, i);
  std::vector<std::vector<QM31>> layers(L + 1);
  layers[0] = codeword;
  FriProof proof;
  proof.params = params;
  std::vector<MerkleTree> trees(L);
  QM31 it = invTwo();
  for (unsigned i = 0; i < L; ++i) {
    size_t ni = layers[i].size(), nn = ni / 2;
    trees[i].init(hashCodeword(layers[i]));
    proof.roots.push_back(trees[i].root());
    ch.absorbDigest(trees[i].root());
    QM31 alpha = ch.sampleQM31();
    std::vector<QM31> next(nn);
    for (size_t j = 0; j < nn; ++j) {
      QM31 y0 = layers[i][j], y1 = layers[i][j + nn];
      QM31 hs = y0.add(y1).mul(it);
      QM31 hd = y0.sub(y1).mul(doms[i][j].inv()).mul(it);
      next[j] = hs.add(alpha.mul(hd));
    }
    layers[i + 1] = std::move(next);
  }
  // fri.zig:228-233 remainder
  size_t rem = (size_t)1 << (params.remainder_log - params.log_blowup);
  std::vector<QM31> xs(doms[L].begin(), doms[L].begin() + rem);
  std::vector<QM31> ys(layers[L].begin(), layers[L].begin() + rem);
  proof.remainder = interpolateLagrange(xs, ys);
  ch.absorbMany(proof.remainder);
  // fri.zig:236-256 queries
  for (uint64_t q = 0; q < params.num_queries; ++q) {
    FriQuery fq;
    uint64_t p0 = ch.sampleIndex(n0);
    fq.index = p0;
    uint64_t p = p0;
    for (unsigned i = 0; i < L; ++i) {
      size_t ni = (size_t)1 << (dlog - i), nn = ni / 2;
      size_t pn = p % nn;
      FriPair pr;
      pr.value0 = layers[i][pn];
      pr.value1 = layers[i][pn + nn];
      pr.path0 = trees[i].open(pn);
      pr.path1 = trees[i].open(pn + nn);
      fq.pairs.push_back(std::move(pr));
      p = pn;
    }
    proof.queries.push_back(std::move(fq));
  }
  if (layers_out) *layers_out = std::move(layers);
  return proof;
}

// fri.zig:135-151.
inline FriProof friProve(const FriParams& params, const std::vector<QM31>& coeffs, Channel& ch) {
  std::vector<QM31> dom0 = friDomainPoints(params, 0);
  std::vector<QM31> ev0(dom0.size());
  for (size_t j = 0; j < dom0.size(); ++j) ev0[j] = evalHorner(coeffs, dom0[j]);
  return friProveCodeword(params, ev0, ch);
}

// fri.zig:277-336.
inline bool friVerify(const FriParams& params, const FriProof& proof, Channel& ch) {
  unsigned L = params.numFoldRounds();
  unsigned dlog = params.domainLogSize();
  size_t n0 = (size_t)1 << dlog;
  if (proof.roots.size() != L) return false;
  if (proof.queries.size() != params.num_queries) return false;
  std::vector<QM31> alphas(L);
  for (unsigned i = 0; i < L; ++i) {
    ch.absorbDigest(proof.roots[i]);
    alphas[i] = ch.sampleQM31();
  }
  ch.absorbMany(proof.remainder);
  for (const auto& q : proof.queries) {
    if (ch.sampleIndex(n0) != q.index) return false;
    if (q.pairs.size() != L) return false;
    uint64_t p = q.index;
    QM31 prev;
    for (unsigned i = 0; i < L; ++i) {
      size_t ni = (size_t)1 << (dlog - i), nn = ni / 2;
      size_t pn = p % nn;
      const FriPair& pr = q.pairs[i];
      if (!merkleVerify(proof.roots[i], pn, hashQM31(pr.value0), pr.path0)) return false;
      if (!merkleVerify(proof.roots[i], pn + nn, hashQM31(pr.value1), pr.path1)) return false;
      if (i > 0) {
        QM31 matched = (p == pn) ? pr.value0 : pr.value1;
        if (!prev.eq(matched)) return false;
      }
      QM31 g = friDomainPoint(params, i, pn);
      QM31 fv = friFoldValue(g, pr.value0, pr.value1, alphas[i]);
      if (i == L - 1) {
        QM31 h = friDomainPoint(params, i + 1, pn);
        if (!evalHorner(proof.remainder, h).eq(fv)) return false;
      }
      prev = fv;
      p = pn;
    }
  }
  return true;
}

}  // namespace orc
