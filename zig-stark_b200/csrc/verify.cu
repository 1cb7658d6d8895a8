// GenericStark(Air).verify (src/m31/stark.zig:660-784) and Fri.verify
// (src/m31/fri.zig:277-336). Like the reference, verification is a host-side replay
// of the transcript plus a few hundred hash and field operations per query; it is
// not on the hot path and runs on the CPU.
#include <memory>
#include <vector>

#include "constraints.cuh"
#include "host.cuh"
#include "verify.cuh"

namespace zs {

namespace {

struct Pair {
  qm31 v0, v1;
  std::vector<Digest> p0, p1;
};
struct FriQuery {
  uint64_t index;
  std::vector<Pair> pairs;
};
struct Reveal {
  uint64_t index;
  std::vector<qm31> values;
  std::vector<std::vector<Digest>> paths;
};
struct Proof {
  StarkParamsH params;
  std::vector<Digest> trace_roots, pre_roots, acc_roots;
  bool has_pre = false, has_acc = false;
  Digest qroot{};
  std::vector<qm31> deep;
  FriParamsH fparams;
  std::vector<Digest> froots;
  std::vector<qm31> remainder;
  std::vector<FriQuery> fq;
  std::vector<Reveal> reveals;
};

Digest rd_digest(WireReader& r) {
  Digest d;
  std::memcpy(d.data(), r.take(32), 32);
  return d;
}
std::vector<Digest> rd_digests(WireReader& r) {
  const uint64_t n = r.len(32);
  std::vector<Digest> v(n);
  for (auto& d : v) d = rd_digest(r);
  return v;
}
std::vector<qm31> rd_qs(WireReader& r) {
  const uint64_t n = r.len(16);
  std::vector<qm31> v(n);
  for (auto& x : v) x = r.q();
  return v;
}

Proof parse(const uint8_t* b, size_t n) {
  WireReader r(b, n);
  Proof p;
  p.params.trace_log = r.u8();
  p.params.log_blowup = r.u8();
  p.params.num_queries = r.u64();
  p.params.remainder_log = r.u8();
  p.trace_roots = rd_digests(r);
  if ((p.has_pre = r.u8() == 1)) p.pre_roots = rd_digests(r);
  if ((p.has_acc = r.u8() == 1)) p.acc_roots = rd_digests(r);
  p.qroot = rd_digest(r);
  p.deep = rd_qs(r);
  p.fparams.log_size = r.u8();
  p.fparams.log_blowup = r.u8();
  p.fparams.num_queries = r.u64();
  p.fparams.remainder_log = r.u8();
  p.froots = rd_digests(r);
  p.remainder = rd_qs(r);
  const uint64_t nq = r.len(16);
  for (uint64_t i = 0; i < nq; ++i) {
    FriQuery q;
    q.index = r.u64();
    const uint64_t np = r.len(32);
    for (uint64_t k = 0; k < np; ++k) {
      Pair pr;
      pr.v0 = r.q();
      pr.v1 = r.q();
      pr.p0 = rd_digests(r);
      pr.p1 = rd_digests(r);
      q.pairs.push_back(std::move(pr));
    }
    p.fq.push_back(std::move(q));
  }
  const uint64_t nr = r.len(24);
  for (uint64_t i = 0; i < nr; ++i) {
    Reveal rv;
    rv.index = r.u64();
    rv.values = rd_qs(r);
    const uint64_t np = r.len(8);
    for (uint64_t k = 0; k < np; ++k) rv.paths.push_back(rd_digests(r));
    p.reveals.push_back(std::move(rv));
  }
  r.end();
  return p;
}

Digest hash_q(const qm31& v) {
  uint32_t o[8];
  b3::hash_qm31(v, o);
  Digest d;
  std::memcpy(d.data(), o, 32);
  return d;
}
Digest hash_pair(const Digest& l, const Digest& r) {
  uint32_t a[8], b[8], o[8];
  std::memcpy(a, l.data(), 32);
  std::memcpy(b, r.data(), 32);
  b3::hash2(a, b, o);
  Digest d;
  std::memcpy(d.data(), o, 32);
  return d;
}
// merkle.zig:72-89.
bool merkle_ok(const Digest& root, uint64_t index, const Digest& leaf, const std::vector<Digest>& path) {
  Digest d = leaf;
  uint64_t idx = index;
  for (const Digest& s : path) {
    d = (idx & 1) == 0 ? hash_pair(d, s) : hash_pair(s, d);
    idx >>= 1;
  }
  return d == root;
}

qm31 fri_point(unsigned dlog, unsigned layer, uint64_t j) {  // fri.zig:96-101
  const qm31 w = q_root_of_unity(dlog - layer);
  return qmul(qpow(q_fri_offset(), (uint64_t)1 << layer), qpow(w, j));
}

// fri.zig:277-336.
bool fri_verify(const FriParamsH& fp, const Proof& p, Channel& ch) {
  const unsigned L = fp.folds(), dlog = fp.domain_log();
  const uint64_t n0 = (uint64_t)1 << dlog;
  if (p.froots.size() != L || p.fq.size() != fp.num_queries) return false;
  std::vector<qm31> alphas(L);
  for (unsigned i = 0; i < L; ++i) {
    ch.absorb(p.froots[i]);
    alphas[i] = ch.sample_q();
  }
  for (auto& v : p.remainder) ch.absorb(v);
  const qm31 inv2 = qfrom_m31(1u << 30);
  for (const FriQuery& q : p.fq) {
    if (ch.sample_index(n0) != q.index) return false;
    if (q.pairs.size() != L) return false;
    uint64_t pos = q.index;
    qm31 prev{};
    for (unsigned i = 0; i < L; ++i) {
      const uint64_t nn = ((uint64_t)1 << (dlog - i)) / 2, pn = pos % nn;
      const Pair& pr = q.pairs[i];
      if (!merkle_ok(p.froots[i], pn, hash_q(pr.v0), pr.p0)) return false;
      if (!merkle_ok(p.froots[i], pn + nn, hash_q(pr.v1), pr.p1)) return false;
      if (i > 0 && !qeq(prev, pos == pn ? pr.v0 : pr.v1)) return false;
      const qm31 g = fri_point(dlog, i, pn);
      const qm31 hs = qmul(qadd(pr.v0, pr.v1), inv2);
      const qm31 hd = qmul(qmul(qsub(pr.v0, pr.v1), qinv(g)), inv2);
      const qm31 fv = qadd(hs, qmul(alphas[i], hd));
      if (i == L - 1) {
        const qm31 h = fri_point(dlog, i + 1, pn);
        if (!qeq(horner(p.remainder.data(), (uint32_t)p.remainder.size(), h), fv)) return false;
      }
      prev = fv;
      pos = pn;
    }
  }
  return true;
}

}  // namespace

bool stark_verify(uint32_t air_id, const uint8_t* params_b, size_t params_len, const uint8_t* pi, size_t pi_len,
                  const uint8_t* proof_b, size_t proof_len, const uint8_t* sep, size_t sep_len) {
  StarkParamsH sp;
  {
    WireReader r(params_b, params_len);
    sp.trace_log = r.u8();
    sp.log_blowup = r.u8();
    sp.num_queries = r.u64();
    sp.remainder_log = r.u8();
    r.end();
  }
  const AirInfo air = make_air(air_id, pi, pi_len);
  const Proof p = parse(proof_b, proof_len);
  const unsigned tl = sp.trace_log, lb = sp.log_blowup, lN = tl + lb;
  if (lN > 30) throw Error(ZS_EMALFORMED, "trace_log + log_blowup above 30");
  const uint64_t n = (uint64_t)1 << tl, N = (uint64_t)1 << lN, shift = (uint64_t)1 << lb;
  const uint32_t m = air.m, n_pre = air.n_pre, n_rel = air.n_rel, m_total = m + n_rel;
  const uint32_t n_deep = 2 * m_total + 1, reveal_len = 2 * m_total + 1 + n_pre;
  const uint32_t total_bound = air.num_bound + n_rel;
  const bool wide = air.id == AIR_ML_LINEAR;  // composed by ml_composition
  if (!wide && (m_total > kMaxCols || air.num_trans > kMaxTrans || total_bound > kMaxBound || n_pre > kMaxPre))
    throw Error(ZS_EGENERIC, "AIR exceeds the compiled-in limits");
  if (air.fixed_n && n != air.fixed_n) throw Error(ZS_EMALFORMED, "the AIR is defined for a fixed trace length");
  if (air.id == AIR_RESCUE_STACKED && n < 8) throw Error(ZS_EMALFORMED, "stacked rescue needs at least 8 rows");
  if (p.trace_roots.size() != m || p.deep.size() != n_deep) return false;
  if (n_pre > 0 && (!p.has_pre || p.pre_roots.size() != n_pre)) return false;
  if (n_rel > 0 && (!p.has_acc || p.acc_roots.size() != n_rel)) return false;
  FriParamsH fp;
  {
    const uint64_t dc = air.max_constraint_degree(n);
    const uint64_t sat = dc > n ? dc - n : 0;
    const uint64_t degree_g = (n - 1) > sat ? (n - 1) : sat;
    unsigned log = 0;
    uint64_t bound = 1;
    while (bound <= degree_g) ++log, bound <<= 1;
    if (log > lN || sp.remainder_log >= lN || sp.remainder_log < lN - log)
      throw Error(ZS_EPROTOCOL, "parameters violate the FRI sizing assertions");
    fp.log_size = (uint8_t)log;
    fp.log_blowup = (uint8_t)(lN - log);
    fp.num_queries = sp.num_queries;
    fp.remainder_log = sp.remainder_log;
  }
  const qm31 w = q_root_of_unity(tl), w_ev = q_root_of_unity(lN);
  Channel ch(sep, sep_len);
  for (auto& d : p.pre_roots) ch.absorb(d);
  for (auto& d : p.trace_roots) ch.absorb(d);
  QuotConsts kc{};
  kc.air = air.consts;
  kc.air.n_div8 = n / 8;
  kc.m = m, kc.m_total = m_total, kc.n_pre = n_pre, kc.num_trans = air.num_trans, kc.n_rel = n_rel;
  kc.total_bound = total_bound;
  kc.last_point = qpow(w, n - 1);
  std::vector<qm31> ac(air.n_lc), ar(n_rel);
  for (auto& a : ac) a = ch.sample_q();
  for (auto& a : ar) a = ch.sample_q();
  for (auto& d : p.acc_roots) ch.absorb(d);
  std::vector<qm31> alphas(air.num_trans + 2 * n_rel);
  for (auto& a : alphas) a = ch.sample_q();
  std::vector<Boundary> bnd;
  air.boundary(n, bnd);
  for (uint32_t r = 0; r < n_rel; ++r) bnd.push_back({m + r, 0, qzero()});
  std::vector<qm31> betas(total_bound);
  for (auto& b : betas) b = ch.sample_q();
  std::unique_ptr<MlConsts> ml;
  if (wide) {
    ml = std::make_unique<MlConsts>();
    for (uint32_t l = 0; l < kMlDim; ++l) ml->ac[l] = ac[l];
    ml->ar = ar[0];
    ml->last_point = kc.last_point;
    ml_set_weights(*ml, air, alphas, betas);
  } else {
    for (uint32_t j = 0; j < air.n_lc; ++j) kc.ac[j] = ac[j];
    for (uint32_t r = 0; r < n_rel; ++r) kc.ar[r] = ar[r];
    for (uint32_t r = 0; r < n_rel; ++r) {
      kc.sel[r] = air.sel[r], kc.mult[r] = air.mult[r], kc.n_keys[r] = air.n_keys[r];
      for (uint32_t j = 0; j < air.n_keys[r]; ++j) kc.keys[r][j] = air.keys[r][j], kc.tabs[r][j] = air.tabs[r][j];
    }
    for (uint32_t t = 0; t < alphas.size(); ++t) kc.alphas[t] = alphas[t];
    for (uint32_t b = 0; b < total_bound; ++b) {
      kc.betas[b] = betas[b];
      kc.b_col[b] = bnd[b].column;
      kc.b_val[b] = bnd[b].value;
      kc.b_pt[b] = qpow(w, bnd[b].step);
    }
    group_boundaries(kc);
    if (const char* bad = quot_consts_out_of_range(kc, 0)) throw Error(ZS_EGENERIC, bad);
  }
  ch.absorb(p.qroot);
  const qm31 z = ch.sample_q();
  for (auto& v : p.deep) ch.absorb(v);
  std::vector<qm31> gammas(n_deep);
  for (auto& g : gammas) g = ch.sample_q();
  if (!fri_verify(fp, p, ch)) return false;
  // stark.zig:713-714 reads one reveal per FRI query and checks only the reveals the
  // proof carries, so the reference accepts a proof with fewer reveals than queries
  // (none at all skips every DEEP and constraint check). This verifier requires exactly
  // one reveal per FRI query; honest proofs always carry that many.
  if (p.reveals.size() != p.fq.size()) return false;
  for (size_t qi = 0; qi < p.reveals.size(); ++qi) {
    const Reveal& rv = p.reveals[qi];
    if (rv.index != p.fq[qi].index) return false;
    if (rv.values.size() != reveal_len || rv.paths.size() != reveal_len) return false;
    const uint64_t p0 = rv.index, pn = (p0 + shift) % N;
    for (uint32_t j = 0; j < m; ++j) {
      if (!merkle_ok(p.trace_roots[j], p0, hash_q(rv.values[j]), rv.paths[j])) return false;
      if (!merkle_ok(p.trace_roots[j], pn, hash_q(rv.values[m_total + j]), rv.paths[m_total + j])) return false;
    }
    for (uint32_t r = 0; r < n_rel; ++r) {
      if (!merkle_ok(p.acc_roots[r], p0, hash_q(rv.values[m + r]), rv.paths[m + r])) return false;
      if (!merkle_ok(p.acc_roots[r], pn, hash_q(rv.values[m_total + m + r]), rv.paths[m_total + m + r])) return false;
    }
    if (!merkle_ok(p.qroot, p0, hash_q(rv.values[2 * m_total]), rv.paths[2 * m_total])) return false;
    for (uint32_t k = 0; k < n_pre; ++k)
      if (!merkle_ok(p.pre_roots[k], p0, hash_q(rv.values[2 * m_total + 1 + k]), rv.paths[2 * m_total + 1 + k]))
        return false;
    const qm31 x0 = qmul(q_fri_offset(), qpow(w_ev, p0));
    const qm31 inv_dz = qinv(qsub(x0, z));
    qm31 g = qzero();
    for (uint32_t j = 0; j < m_total; ++j) {
      g = qadd(g, qmul(gammas[j], qmul(qsub(rv.values[j], p.deep[j]), inv_dz)));
      g = qadd(g, qmul(gammas[m_total + j], qmul(qsub(rv.values[m_total + j], p.deep[m_total + j]), inv_dz)));
    }
    g = qadd(g, qmul(gammas[2 * m_total], qmul(qsub(rv.values[2 * m_total], p.deep[2 * m_total]), inv_dz)));
    if (p.fq[qi].pairs.empty()) return false;
    const uint64_t p1 = p0 % (N / 2);
    const qm31 leaf = p0 == p1 ? p.fq[qi].pairs[0].v0 : p.fq[qi].pairs[0].v1;
    if (!qeq(g, leaf)) return false;
    const qm31 zh = qsub(qpow(x0, n), qone());
    const qm31* vals = rv.values.data();
    const qm31 h = wide ? ml_composition(*ml, x0, vals, vals + m_total, vals + 2 * m_total + 1, zh, false)
                        : composition(kc, x0, vals, vals + m_total, vals + 2 * m_total + 1, zh);
    if (!qeq(h, qmul(zh, rv.values[2 * m_total]))) return false;
  }
  return true;
}

}  // namespace zs
