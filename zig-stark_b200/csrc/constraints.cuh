// Constraint composition of GenericStark (src/m31/stark.zig:243-297, 505-533),
// shared by the device quotient kernel, the host-side Q(z) and the verifier.
#pragma once
#include "airs.cuh"

namespace zs {

// Everything the quotient and DEEP kernels need beyond the codewords.
struct QuotConsts {
  AirConsts air;
  uint32_t m, m_total, n_pre, num_trans, n_rel, total_bound, shift;
  unsigned log_N, log_blowup;
  qm31 last_point;  // w^(n-1)
  qm31 offset;      // FRI_OFFSET
  qm31 alphas[kMaxTrans + 2 * kMaxRel];
  qm31 betas[kMaxBound];
  uint32_t b_col[kMaxBound];
  qm31 b_val[kMaxBound];
  qm31 b_pt[kMaxBound];  // p_k = w^step_k
  qm31 zh[8], zh_inv[8];  // Z_H(d_i) depends on i mod 2^log_blowup
  qm31 ac[kMaxKey], ar[kMaxRel];
  uint32_t sel[kMaxRel], mult[kMaxRel], n_keys[kMaxRel], keys[kMaxRel][kMaxKey], tabs[kMaxRel][kMaxKey];
};

__device__ __host__ __forceinline__ qm31 combined_key(const qm31* ac, uint32_t nk, const uint32_t* cols,
                                                      const qm31* row) {
  qm31 key = qzero();
  for (uint32_t j = 0; j < nk; ++j) key = qadd(key, qmul(ac[j], row[cols[j]]));
  return key;
}

// stark.zig:259-276 (denominator-cleared LogUp constraint).
__device__ __host__ __forceinline__ qm31 lookup_constraint(const QuotConsts& k, uint32_t r, const qm31* cur,
                                                           const qm31* pre, const qm31& acc, const qm31& accn) {
  const qm31 sel = cur[k.sel[r]], mult = cur[k.mult[r]];
  const qm31 key = combined_key(k.ac, k.n_keys[r], k.keys[r], cur);
  const qm31 tkey = combined_key(k.ac, k.n_keys[r], k.tabs[r], pre);
  const qm31 dacc = qsub(accn, acc);
  const qm31 lb = qsub(qmul(dacc, qsub(k.ar[r], key)), mult);
  const qm31 tb = qadd(qmul(dacc, qsub(k.ar[r], tkey)), qone());
  return qadd(qmul(sel, lb), qmul(qsub(qone(), sel), tb));
}

// Hc(x) (stark.zig:505-533): transitions x (x - w^(n-1)), cyclic LogUp and
// selector-binarity constraints, boundary terms with Z_H(x) / (x - p_k).
__device__ __host__ inline qm31 composition(const QuotConsts& k, const qm31& x, const qm31* cur, const qm31* next,
                                            const qm31* pre, const qm31& zh) {
  qm31 res[kMaxTrans];
  air_eval(k.air, x, cur, next, res);
  qm31 h = qzero();
  const qm31 xl = qsub(x, k.last_point);
  for (uint32_t t = 0; t < k.num_trans; ++t) h = qadd(h, qmul(k.alphas[t], qmul(res[t], xl)));
  for (uint32_t r = 0; r < k.n_rel; ++r)
    h = qadd(h, qmul(k.alphas[k.num_trans + r], lookup_constraint(k, r, cur, pre, cur[k.m + r], next[k.m + r])));
  for (uint32_t r = 0; r < k.n_rel; ++r) {
    const qm31 sel = cur[k.sel[r]];
    h = qadd(h, qmul(k.alphas[k.num_trans + k.n_rel + r], qmul(sel, qsub(qone(), sel))));
  }
  for (uint32_t b = 0; b < k.total_bound; ++b) {
    const qm31 term = qmul(qmul(qsub(cur[k.b_col[b]], k.b_val[b]), zh), qinv(qsub(x, k.b_pt[b])));
    h = qadd(h, qmul(k.betas[b], term));
  }
  return h;
}

}  // namespace zs
