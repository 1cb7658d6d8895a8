// ORACLE — test infrastructure only. GenericStark(Air) restated from
// src/m31/stark.zig:
//   compositionLogSize 197-204, maxConstraintDegree 217-221, friParams 226-239,
//   combinedKey 243-247, lookupConstraintAt 259-276, rowContribution 283-297,
//   proveWithPreprocessed 327-658, verify 660-784, computeQuotientAt 794-849.
//
// `Mode::Lagrange` runs the reference's own O(n^2) interpolation and O(n*N)
// Horner evaluation. `Mode::Ntt` swaps in the radix-2 NTT for those two steps
// only; everything else (transcript order, quotient, DEEP, FRI, queries) is the
// same code. Both produce the same bytes (asserted in the tests at every size
// where Lagrange finishes), so the NTT mode carries parity to larger traces.
#pragma once
#include <vector>

#include "airs.hpp"
#include "fri.hpp"

namespace orc {

enum class Mode { Lagrange = 0, Ntt = 1 };

struct Stark {
  const Air& air;
  size_t m, num_trans, num_bound, n_pre, n_lc, n_rel, m_total, n_trans_total, total_bound,
      n_deep, reveal_len;

  explicit Stark(const Air& a) : air(a) {
    m = air.num_columns;
    num_trans = air.num_transitions;
    num_bound = air.num_boundary;
    n_pre = air.num_preprocessed;
    n_lc = air.num_lookup_columns;
    n_rel = air.num_lookup_relations;
    m_total = m + n_rel;
    n_trans_total = num_trans + 2 * n_rel;
    total_bound = num_bound + n_rel;
    n_deep = 2 * m_total + 1;
    reveal_len = 2 * m_total + 1 + n_pre;
  }

  size_t maxConstraintDegree(size_t n) const {  // stark.zig:217-221
    size_t ad = air.maxConstraintDegree(n);
    size_t ld = n_rel > 0 ? 3 * (n - 1) : 0;
    return ad > ld ? ad : ld;
  }
  unsigned compositionLogSize(size_t n) const {  // stark.zig:197-204
    size_t dc = maxConstraintDegree(n);
    size_t sat = dc > n ? dc - n : 0;
    size_t degree_g = (n - 1) > sat ? (n - 1) : sat;
    unsigned log = 0;
    size_t bound = 1;
    while (bound <= degree_g) {
      ++log;
      bound <<= 1;
    }
    return log;
  }
  FriParams friParams(const StarkParams& p) const {  // stark.zig:226-239
    size_t n = p.traceLen();
    unsigned log_size = compositionLogSize(n);
    unsigned domain_log = p.trace_log + p.log_blowup;
    if (log_size > domain_log || p.remainder_log >= domain_log ||
        p.remainder_log < domain_log - log_size)
      throw WireError("parameters violate the FRI sizing assertions", -4);
    FriParams f;
    f.log_size = (uint8_t)log_size;
    f.log_blowup = (uint8_t)(domain_log - log_size);
    f.num_queries = p.num_queries;
    f.remainder_log = p.remainder_log;
    return f;
  }

  QM31 combinedKey(const std::vector<size_t>& cols, const std::vector<QM31>& ac,
                   const QM31* row) const {
    QM31 k = QM31::zero();
    for (size_t j = 0; j < cols.size(); ++j) k = k.add(ac[j].mul(row[cols[j]]));
    return k;
  }
  QM31 lookupConstraintAt(size_t r, const std::vector<QM31>& ac, const std::vector<QM31>& ar,
                          const QM31* row, const QM31* pre, QM31 acc, QM31 accn) const {
    QM31 sel = row[air.selector_cols[r]];
    QM31 mult = row[air.mult_cols[r]];
    QM31 key = combinedKey(air.key_cols[r], ac, row);
    QM31 tkey = combinedKey(air.table_cols[r], ac, pre);
    QM31 dacc = accn.sub(acc);
    QM31 lb = dacc.mul(ar[r].sub(key)).sub(mult);
    QM31 tb = dacc.mul(ar[r].sub(tkey)).add(QM31::one());
    return sel.mul(lb).add(QM31::one().sub(sel).mul(tb));
  }
  QM31 rowContribution(size_t r, const std::vector<QM31>& ac, const std::vector<QM31>& ar,
                       const QM31* row, const QM31* pre) const {
    QM31 sel = row[air.selector_cols[r]];
    QM31 mult = row[air.mult_cols[r]];
    QM31 key = combinedKey(air.key_cols[r], ac, row);
    QM31 tkey = combinedKey(air.table_cols[r], ac, pre);
    QM31 lt = sel.mul(mult.mul(ar[r].sub(key).inv()));
    QM31 tt = QM31::one().sub(sel).mul(ar[r].sub(tkey).inv());
    return lt.sub(tt);
  }

  // Interpolate on H and evaluate on D, in the selected mode.
  void lde(const std::vector<QM31>& col, const StarkParams& p, const std::vector<QM31>& h_points,
           const std::vector<QM31>& d_points, Mode mode, std::vector<QM31>& coeffs,
           std::vector<QM31>& codeword) const {
    if (mode == Mode::Lagrange) {
      coeffs = interpolateLagrange(h_points, col);
      codeword.resize(d_points.size());
      for (size_t i = 0; i < d_points.size(); ++i) codeword[i] = evalHorner(coeffs, d_points[i]);
    } else {
      coeffs = interpolateSubgroupNtt(col, p.trace_log);
      codeword = evaluateCosetNtt(coeffs, friOffset(), p.trace_log + p.log_blowup);
    }
  }

  // Composition value Hc at one point (shared by the quotient loop and
  // computeQuotientAt). `cur`/`next` have m_total entries, `pre` n_pre.
  QM31 composition(const QM31& x, const QM31* cur, const QM31* next, const QM31* pre,
                   const QM31& last_point, const QM31& zh, const std::vector<QM31>& alphas,
                   const std::vector<QM31>& betas, const std::vector<BoundaryAssertion>& bnd,
                   const std::vector<QM31>& ac, const std::vector<QM31>& ar, const QM31& w,
                   const std::vector<QM31>* inv_dp) const {
    std::vector<QM31> res(num_trans);
    air.evalTransition(x, cur, next, res.data());
    QM31 h = QM31::zero();
    for (size_t k = 0; k < num_trans; ++k) h = h.add(alphas[k].mul(res[k].mul(x.sub(last_point))));
    for (size_t r = 0; r < n_rel; ++r) {
      QM31 c = lookupConstraintAt(r, ac, ar, cur, pre, cur[m + r], next[m + r]);
      h = h.add(alphas[num_trans + r].mul(c));
    }
    for (size_t r = 0; r < n_rel; ++r) {
      QM31 sel = cur[air.selector_cols[r]];
      h = h.add(alphas[num_trans + n_rel + r].mul(sel.mul(QM31::one().sub(sel))));
    }
    for (size_t k = 0; k < total_bound; ++k) {
      QM31 inv;
      if (inv_dp) {
        inv = (*inv_dp)[k];
      } else {
        QM31 pk = w.pow(bnd[k].step);
        inv = x.sub(pk).inv();
      }
      QM31 term = cur[bnd[k].column].sub(bnd[k].value).mul(zh).mul(inv);
      h = h.add(betas[k].mul(term));
    }
    return h;
  }

  // stark.zig:327-658.
  StarkProof prove(const StarkParams& params, const std::vector<std::vector<QM31>>& pre,
                   const std::vector<std::vector<QM31>>& trace, Channel& ch, Mode mode) const {
    const size_t n = params.traceLen(), N = params.domainLen(), shift = params.shift();
    air.checkTraceLen(n);
    if (trace.size() != m || pre.size() != n_pre) throw WireError("column count mismatch", -2);
    for (auto& c : trace)
      if (c.size() != n) throw WireError("column length mismatch", -2);
    for (auto& c : pre)
      if (c.size() != n) throw WireError("column length mismatch", -2);
    FriParams fparams = friParams(params);

    QM31 w = QM31::primitiveRootOfUnity(params.trace_log);
    QM31 w_ev = QM31::primitiveRootOfUnity(params.trace_log + params.log_blowup);
    std::vector<QM31> h_points(n);
    h_points[0] = QM31::one();
    for (size_t i = 1; i < n; ++i) h_points[i] = h_points[i - 1].mul(w);
    std::vector<QM31> d_points(N);
    d_points[0] = friOffset();
    for (size_t i = 1; i < N; ++i) d_points[i] = d_points[i - 1].mul(w_ev);

    std::vector<std::vector<QM31>> coeffs(m_total), codewords(m_total);
    std::vector<std::vector<QM31>> pre_coeffs(n_pre), pre_cw(n_pre);
    // columns are independent until their roots are absorbed: LDE and tree per column in
    // parallel, then the roots in the reference's order
    std::vector<MerkleTree> pre_trees(n_pre), trace_trees(m), acc_trees(n_rel);
#pragma omp parallel for schedule(dynamic)
    for (long jj = 0; jj < (long)(m + n_pre); ++jj) {
      const size_t j = (size_t)jj;
      if (j < m) {
        lde(trace[j], params, h_points, d_points, mode, coeffs[j], codewords[j]);
        trace_trees[j].init(hashCodeword(codewords[j]));
      } else {
        const size_t k = j - m;
        lde(pre[k], params, h_points, d_points, mode, pre_coeffs[k], pre_cw[k]);
        pre_trees[k].init(hashCodeword(pre_cw[k]));
      }
    }

    StarkProof proof;
    proof.params = params;
    if (n_pre > 0) proof.preprocessed_roots = std::vector<Digest>();
    for (size_t j = 0; j < n_pre; ++j) {
      proof.preprocessed_roots->push_back(pre_trees[j].root());
      ch.absorbDigest(pre_trees[j].root());
    }
    for (size_t j = 0; j < m; ++j) {
      proof.trace_roots.push_back(trace_trees[j].root());
      ch.absorbDigest(trace_trees[j].root());
    }
    std::vector<QM31> ac(n_lc), ar(n_rel);
    for (auto& a : ac) a = ch.sampleQM31();
    for (auto& a : ar) a = ch.sampleQM31();

    // stark.zig:429-446 accumulator fill on H
    std::vector<std::vector<QM31>> acc_h(n_rel, std::vector<QM31>(n));
    std::vector<QM31> hrow(m), hpre(n_pre);
    for (size_t r = 0; r < n_rel; ++r) acc_h[r][0] = QM31::zero();
    for (size_t i = 1; i < n; ++i) {
      for (size_t j = 0; j < m; ++j) hrow[j] = trace[j][i - 1];
      for (size_t j = 0; j < n_pre; ++j) hpre[j] = pre[j][i - 1];
      for (size_t r = 0; r < n_rel; ++r)
        acc_h[r][i] = acc_h[r][i - 1].add(rowContribution(r, ac, ar, hrow.data(), hpre.data()));
    }
    if (n_rel > 0) proof.accumulator_roots = std::vector<Digest>();
    for (size_t r = 0; r < n_rel; ++r) {
      lde(acc_h[r], params, h_points, d_points, mode, coeffs[m + r], codewords[m + r]);
      acc_trees[r].init(hashCodeword(codewords[m + r]));
      proof.accumulator_roots->push_back(acc_trees[r].root());
      ch.absorbDigest(acc_trees[r].root());
    }

    std::vector<QM31> alphas(n_trans_total);
    for (auto& a : alphas) a = ch.sampleQM31();
    std::vector<BoundaryAssertion> bnd(total_bound);
    air.boundaryAssertions(n, bnd.data());
    for (size_t r = 0; r < n_rel; ++r) bnd[num_bound + r] = {m + r, 0, QM31::zero()};
    std::vector<QM31> betas(total_bound);
    for (auto& b : betas) b = ch.sampleQM31();

    // stark.zig:484-536 quotient on D
    std::vector<QM31> q(N);
    {
      QM31 last_point = h_points[n - 1];
      std::vector<QM31> pks(total_bound);
      for (size_t k = 0; k < total_bound; ++k) pks[k] = w.pow(bnd[k].step);
      // every point is independent; the loop body is the reference's per point
#pragma omp parallel for schedule(static)
      for (long ii = 0; ii < (long)N; ++ii) {
        const size_t i = (size_t)ii;
        std::vector<QM31> cur(m_total), nxt(m_total), rp(n_pre), inv_dp(total_bound);
        QM31 zh = d_points[i].pow(n).sub(QM31::one());
        QM31 inv_zh = zh.inv();
        for (size_t j = 0; j < m_total; ++j) {
          cur[j] = codewords[j][i];
          nxt[j] = codewords[j][(i + shift) % N];
        }
        for (size_t j = 0; j < n_pre; ++j) rp[j] = pre_cw[j][i];
        for (size_t k = 0; k < total_bound; ++k) inv_dp[k] = d_points[i].sub(pks[k]).inv();
        QM31 h = composition(d_points[i], cur.data(), nxt.data(), rp.data(), last_point, zh, alphas,
                             betas, bnd, ac, ar, w, &inv_dp);
        q[i] = h.mul(inv_zh);
      }
    }
    MerkleTree qtree(hashCodeword(q));
    proof.quotient_root = qtree.root();
    ch.absorbDigest(qtree.root());

    QM31 z = ch.sampleQM31();
    QM31 wz = z.mul(w);
    proof.deep_evals.resize(n_deep);
    for (size_t j = 0; j < m_total; ++j) {
      proof.deep_evals[j] = evalHorner(coeffs[j], z);
      proof.deep_evals[m_total + j] = evalHorner(coeffs[j], wz);
    }
    proof.deep_evals[2 * m_total] = quotientAt(z, coeffs, pre_coeffs, n, w, alphas, betas, bnd, ac, ar);
    ch.absorbMany(proof.deep_evals);
    std::vector<QM31> gammas(n_deep);
    for (auto& g : gammas) g = ch.sampleQM31();

    // stark.zig:577-588 DEEP codeword
    std::vector<QM31> g(N);
#pragma omp parallel for schedule(static)
    for (long ii = 0; ii < (long)N; ++ii) {
      const size_t i = (size_t)ii;
      QM31 inv_dz = d_points[i].sub(z).inv();
      QM31 gv = QM31::zero();
      for (size_t j = 0; j < m_total; ++j) {
        gv = gv.add(gammas[j].mul(codewords[j][i].sub(proof.deep_evals[j]).mul(inv_dz)));
        gv = gv.add(gammas[m_total + j].mul(
            codewords[j][(i + shift) % N].sub(proof.deep_evals[m_total + j]).mul(inv_dz)));
      }
      gv = gv.add(gammas[2 * m_total].mul(q[i].sub(proof.deep_evals[2 * m_total]).mul(inv_dz)));
      g[i] = gv;
    }
    proof.fri = friProveCodeword(fparams, g, ch);

    // stark.zig:595-625 reveals
    for (uint64_t qi = 0; qi < params.num_queries; ++qi) {
      QueryReveal rv;
      uint64_t p0 = proof.fri.queries[qi].index;
      rv.query_index = p0;
      size_t pn = (p0 + shift) % N;
      rv.values.resize(reveal_len);
      rv.paths.resize(reveal_len);
      for (size_t j = 0; j < m; ++j) {
        rv.values[j] = codewords[j][p0];
        rv.paths[j] = trace_trees[j].open(p0);
        rv.values[m_total + j] = codewords[j][pn];
        rv.paths[m_total + j] = trace_trees[j].open(pn);
      }
      for (size_t r = 0; r < n_rel; ++r) {
        rv.values[m + r] = codewords[m + r][p0];
        rv.paths[m + r] = acc_trees[r].open(p0);
        rv.values[m_total + m + r] = codewords[m + r][pn];
        rv.paths[m_total + m + r] = acc_trees[r].open(pn);
      }
      rv.values[2 * m_total] = q[p0];
      rv.paths[2 * m_total] = qtree.open(p0);
      for (size_t k = 0; k < n_pre; ++k) {
        rv.values[2 * m_total + 1 + k] = pre_cw[k][p0];
        rv.paths[2 * m_total + 1 + k] = pre_trees[k].open(p0);
      }
      proof.queries.push_back(std::move(rv));
    }
    return proof;
  }

  // stark.zig:794-849.
  QM31 quotientAt(const QM31& z, const std::vector<std::vector<QM31>>& coeffs,
                  const std::vector<std::vector<QM31>>& pre_coeffs, size_t n, const QM31& w,
                  const std::vector<QM31>& alphas, const std::vector<QM31>& betas,
                  const std::vector<BoundaryAssertion>& bnd, const std::vector<QM31>& ac,
                  const std::vector<QM31>& ar) const {
    std::vector<QM31> cur(m_total), nxt(m_total), rp(n_pre);
    for (size_t j = 0; j < m_total; ++j) {
      cur[j] = evalHorner(coeffs[j], z);
      nxt[j] = evalHorner(coeffs[j], z.mul(w));
    }
    for (size_t j = 0; j < n_pre; ++j) rp[j] = evalHorner(pre_coeffs[j], z);
    QM31 last_point = w.pow(n - 1);
    QM31 zh = z.pow(n).sub(QM31::one());
    QM31 h = composition(z, cur.data(), nxt.data(), rp.data(), last_point, zh, alphas, betas, bnd, ac,
                         ar, w, nullptr);
    return h.mul(zh.inv());
  }

  // stark.zig:660-784.
  bool verify(const StarkParams& params, const StarkProof& proof, Channel& ch) const {
    const size_t n = params.traceLen(), N = params.domainLen(), shift = params.shift();
    air.checkTraceLen(n);
    if (proof.trace_roots.size() != m) return false;
    if (proof.deep_evals.size() != n_deep) return false;
    if (n_pre > 0 && (!proof.preprocessed_roots || proof.preprocessed_roots->size() != n_pre)) return false;
    if (n_rel > 0 && (!proof.accumulator_roots || proof.accumulator_roots->size() != n_rel)) return false;
    // The reference iterates proof.queries and indexes fri.queries[qi] (stark.zig:713-714);
    // more reveals than FRI queries would index past the end there.
    if (proof.queries.size() > proof.fri.queries.size()) return false;
    FriParams fparams = friParams(params);
    QM31 w = QM31::primitiveRootOfUnity(params.trace_log);
    QM31 w_ev = QM31::primitiveRootOfUnity(params.trace_log + params.log_blowup);
    for (size_t k = 0; k < n_pre; ++k) ch.absorbDigest((*proof.preprocessed_roots)[k]);
    for (size_t j = 0; j < m; ++j) ch.absorbDigest(proof.trace_roots[j]);
    std::vector<QM31> ac(n_lc), ar(n_rel);
    for (auto& a : ac) a = ch.sampleQM31();
    for (auto& a : ar) a = ch.sampleQM31();
    for (size_t r = 0; r < n_rel; ++r) ch.absorbDigest((*proof.accumulator_roots)[r]);
    std::vector<QM31> alphas(n_trans_total);
    for (auto& a : alphas) a = ch.sampleQM31();
    std::vector<BoundaryAssertion> bnd(total_bound);
    air.boundaryAssertions(n, bnd.data());
    for (size_t r = 0; r < n_rel; ++r) bnd[num_bound + r] = {m + r, 0, QM31::zero()};
    std::vector<QM31> betas(total_bound);
    for (auto& b : betas) b = ch.sampleQM31();
    ch.absorbDigest(proof.quotient_root);
    QM31 z = ch.sampleQM31();
    ch.absorbMany(proof.deep_evals);
    std::vector<QM31> gammas(n_deep);
    for (auto& g : gammas) g = ch.sampleQM31();
    if (!friVerify(fparams, proof.fri, ch)) return false;
    QM31 last_point = w.pow(n - 1);
    for (size_t qi = 0; qi < proof.queries.size(); ++qi) {
      const QueryReveal& qv = proof.queries[qi];
      if (qv.query_index != proof.fri.queries[qi].index) return false;
      if (qv.values.size() != reveal_len || qv.paths.size() != reveal_len) return false;
      uint64_t p0 = qv.query_index;
      size_t pn = (p0 + shift) % N;
      for (size_t j = 0; j < m; ++j) {
        if (!merkleVerify(proof.trace_roots[j], p0, hashQM31(qv.values[j]), qv.paths[j])) return false;
        if (!merkleVerify(proof.trace_roots[j], pn, hashQM31(qv.values[m_total + j]), qv.paths[m_total + j]))
          return false;
      }
      for (size_t r = 0; r < n_rel; ++r) {
        if (!merkleVerify((*proof.accumulator_roots)[r], p0, hashQM31(qv.values[m + r]), qv.paths[m + r]))
          return false;
        if (!merkleVerify((*proof.accumulator_roots)[r], pn, hashQM31(qv.values[m_total + m + r]),
                          qv.paths[m_total + m + r]))
          return false;
      }
      if (!merkleVerify(proof.quotient_root, p0, hashQM31(qv.values[2 * m_total]), qv.paths[2 * m_total]))
        return false;
      for (size_t k = 0; k < n_pre; ++k)
        if (!merkleVerify((*proof.preprocessed_roots)[k], p0, hashQM31(qv.values[2 * m_total + 1 + k]),
                          qv.paths[2 * m_total + 1 + k]))
          return false;
      QM31 x0 = friOffset().mul(w_ev.pow(p0));
      QM31 inv_dz = x0.sub(z).inv();
      QM31 gv = QM31::zero();
      for (size_t j = 0; j < m_total; ++j) {
        gv = gv.add(gammas[j].mul(qv.values[j].sub(proof.deep_evals[j]).mul(inv_dz)));
        gv = gv.add(gammas[m_total + j].mul(qv.values[m_total + j].sub(proof.deep_evals[m_total + j]).mul(inv_dz)));
      }
      gv = gv.add(gammas[2 * m_total].mul(qv.values[2 * m_total].sub(proof.deep_evals[2 * m_total]).mul(inv_dz)));
      size_t n1 = N / 2, p1 = p0 % n1;
      if (proof.fri.queries[qi].pairs.empty()) return false;
      const FriPair& pair0 = proof.fri.queries[qi].pairs[0];
      QM31 leaf = (p0 == p1) ? pair0.value0 : pair0.value1;
      if (!gv.eq(leaf)) return false;
      const QM31* cur = qv.values.data();
      const QM31* nxt = qv.values.data() + m_total;
      const QM31* rp = qv.values.data() + 2 * m_total + 1;
      QM31 zh = x0.pow(n).sub(QM31::one());
      QM31 h = composition(x0, cur, nxt, rp, last_point, zh, alphas, betas, bnd, ac, ar, w, nullptr);
      if (!h.eq(zh.mul(qv.values[2 * m_total]))) return false;
    }
    return true;
  }
};

}  // namespace orc
