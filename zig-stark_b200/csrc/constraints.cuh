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
  uint32_t n_bpts;         // distinct boundary points, bpts[g], and b_grp[b] = g with bpts[g] = b_pt[b]
  uint32_t b_grp[kMaxBound];
  qm31 bpts[kMaxBound];
  uint32_t per_mask;  // stacked Rescue: row i & per_mask of the periodic table (a device
                      // buffer of 8 * 2^log_blowup rows of 5 values, airs.cuh) holds the
                      // periodic values of domain point i
  qm31 on;            // FRI_OFFSET^n: Z_H(d_i) = on * w_(2^log_blowup)^(i mod 2^log_blowup) - 1,
                      // kept in a device table of 2^log_blowup (Z_H, Z_H^-1) pairs
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

// Composition constants of the linear-layer AIR (AIR_ML_LINEAR, airs.cuh), whose 259
// committed columns are streamed by its own kernels instead of held per thread.
// Hc(x) (stark.zig:505-533) for this AIR is
//   (x - w^(n-1)) sum_k alpha_k (y_k - sum_l W[k][l] x_l)
//     + alpha_look L(x) + alpha_bin sel (1 - sel)
//     + Z_H(x) (beta_sel sel / (x - w^(n-1)) + beta_acc acc / (x - 1)),
// L the denominator-cleared LogUp constraint (stark.zig:259-276) of the key
// sum_l ac_l x_l against the table key sum_l ac_l P_l. The transition sum is taken as
// sum_k alpha_k y_k - sum_l beta_l x_l with beta_l = sum_k alpha_k W[k][l]: equal in the
// ring, and 2 * 128 products per point instead of 128 * 129.
struct MlConsts {
  qm31 ac[kMlDim];       // LogUp column challenges
  qm31 alpha_y[kMlDim];  // transition weights alpha_k
  qm31 beta_x[kMlDim];   // sum_k alpha_k W[k][l]
  qm31 ar, alpha_look, alpha_bin, beta_sel, beta_acc;
  qm31 last_point;  // w^(n-1), also the point of the sel boundary
  qm31 offset;      // FRI_OFFSET
  uint32_t log_N, log_blowup, shift;
};

// The composition at x from the row's values: cur/next index the m_total = kMlCols + 1
// main and accumulator columns, pre the kMlDim preprocessed ones. `units`: x - w^(n-1)
// and x - 1 are units (always on the evaluation domain), so both inverses come from one.
__device__ __host__ inline qm31 ml_composition(const MlConsts& k, const qm31& x, const qm31* cur, const qm31* next,
                                               const qm31* pre, const qm31& zh, bool units) {
  qm31 ty = qzero(), tx = qzero(), key = qzero(), tkey = qzero();
  for (uint32_t l = 0; l < kMlDim; ++l) {
    ty = qadd(ty, qmul(k.alpha_y[l], cur[kMlDim + l]));
    tx = qadd(tx, qmul(k.beta_x[l], cur[l]));
    key = qadd(key, qmul(k.ac[l], cur[l]));
    tkey = qadd(tkey, qmul(k.ac[l], pre[l]));
  }
  const qm31 sel = cur[kMlSel], mult = cur[kMlMult], acc = cur[kMlCols], accn = next[kMlCols];
  qm31 h = qmul(qsub(ty, tx), qsub(x, k.last_point));
  const qm31 dacc = qsub(accn, acc);
  const qm31 lb = qsub(qmul(dacc, qsub(k.ar, key)), mult);
  const qm31 tb = qadd(qmul(dacc, qsub(k.ar, tkey)), qone());
  h = qadd(h, qmul(k.alpha_look, qadd(qmul(sel, lb), qmul(qsub(qone(), sel), tb))));
  h = qadd(h, qmul(k.alpha_bin, qmul(sel, qsub(qone(), sel))));
  const qm31 d_sel = qsub(x, k.last_point), d_acc = qsub(x, qone());
  qm31 i_sel, i_acc;
  if (units) {
    const qm31 inv = qinv(qmul(d_sel, d_acc));
    i_sel = qmul(inv, d_acc);
    i_acc = qmul(inv, d_sel);
  } else {
    i_sel = qinv(d_sel);
    i_acc = qinv(d_acc);
  }
  const qm31 b = qadd(qmul(k.beta_sel, qmul(sel, i_sel)), qmul(k.beta_acc, qmul(acc, i_acc)));
  return qadd(h, qmul(b, zh));
}

// Fills the linear-layer AIR's weights from the sampled transition weights (128
// transitions, then the LogUp and selector-binarity constraints) and boundary weights
// (sel at w^(n-1), then acc at 1): beta_l = sum_k alpha_k W[k][l].
inline void ml_set_weights(MlConsts& k, const AirInfo& air, const std::vector<qm31>& alphas,
                           const std::vector<qm31>& betas) {
  for (uint32_t l = 0; l < kMlDim; ++l) {
    k.alpha_y[l] = alphas[l];
    k.beta_x[l] = qzero();
  }
  for (uint32_t r = 0; r < kMlDim; ++r)
    for (uint32_t l = 0; l < kMlDim; ++l) k.beta_x[l] = qadd(k.beta_x[l], qmul_m(alphas[r], air.w[(size_t)r * kMlDim + l]));
  k.alpha_look = alphas[kMlDim];
  k.alpha_bin = alphas[kMlDim + 1];
  k.beta_sel = betas[0];
  k.beta_acc = betas[1];
}

// Columns an AIR's transition constraints read from `current` / `next` (air_eval).
inline uint32_t air_columns_read(uint32_t id) {
  switch (id) {
    case AIR_FIB:
    case AIR_SEEDED_FIB: return 2;
    case AIR_RESCUE_EXAMPLE: return 4;
    case AIR_RESCUE_STACKED: return 12;
    case AIR_LINEAR_EXAMPLE: return 1;
    default: return 0;
  }
}

// Host-side check, before every launch that reads `k`, that each index the quotient,
// LogUp and DEEP kernels take from it stays inside the arrays it selects from: the
// per-thread column arrays (m_total main + accumulator columns, n_pre preprocessed),
// the boundary groups, the periodic table and the Z_H table (`zh_entries` pairs; 0 for
// the host-side evaluation, which reads no table). `lookups_only`: the accumulator
// phase, before the boundaries are filled in. Returns a message naming the first index
// out of range, or nullptr.
inline const char* quot_consts_out_of_range(const QuotConsts& k, uint32_t zh_entries, bool lookups_only = false) {
  if (k.m_total > kMaxCols || k.n_pre > kMaxPre || k.m + k.n_rel != k.m_total) return "column counts";
  if (k.num_trans > kMaxTrans || k.n_rel > kMaxRel || k.total_bound > kMaxBound) return "constraint counts";
  if (air_columns_read(k.air.id) > k.m) return "transition columns";
  for (uint32_t r = 0; r < k.n_rel; ++r) {
    if (k.sel[r] >= k.m || k.mult[r] >= k.m) return "lookup selector or multiplicity column";
    if (k.n_keys[r] > kMaxKey) return "lookup key count";
    for (uint32_t j = 0; j < k.n_keys[r]; ++j)
      if (k.keys[r][j] >= k.m || k.tabs[r][j] >= k.n_pre) return "lookup key or table column";
  }
  if (lookups_only) return nullptr;
  if (k.n_bpts > k.total_bound) return "boundary groups";
  for (uint32_t b = 0; b < k.total_bound; ++b) {
    if (k.b_col[b] >= k.m_total) return "boundary column";
    if (k.b_grp[b] >= k.n_bpts) return "boundary group";
  }
  if (zh_entries == 0) return nullptr;  // host-side evaluation: no tables
  if (k.air.id == AIR_RESCUE_STACKED && (uint64_t)k.per_mask + 1 != (8ull << k.log_blowup)) return "periodic table";
  if (((uint64_t)1 << k.log_blowup) != zh_entries) return "vanishing-polynomial table";
  return nullptr;
}

// Groups the boundary assertions by their point (host side, after b_pt is filled).
inline void group_boundaries(QuotConsts& k) {
  k.n_bpts = 0;
  for (uint32_t b = 0; b < k.total_bound; ++b) {
    uint32_t g = 0;
    while (g < k.n_bpts && !qeq(k.bpts[g], k.b_pt[b])) ++g;
    if (g == k.n_bpts) k.bpts[k.n_bpts++] = k.b_pt[b];
    k.b_grp[b] = g;
  }
}

// Hc(x) (stark.zig:505-533): transitions x (x - w^(n-1)), cyclic LogUp and
// selector-binarity constraints, boundary terms with Z_H(x) / (x - p_k). `per`: the
// periodic values of the stacked Rescue AIR at x (rescue_stacked_eval in airs.cuh).
// Evaluated as sum_t alpha_t C_t(x) (x - w^(n-1)) = (x - w^(n-1)) sum_t alpha_t C_t(x) and
// sum_k beta_k (f_k(x) - v_k) Z_H(x) / (x - p_k) = Z_H(x) sum_p (1 / (x - p)) sum_{k: p_k = p}
// beta_k (f_k(x) - v_k): equal in the ring by distributivity, with one inverse per
// distinct boundary point. `units`: every x - p is a unit (true on the evaluation domain,
// whose offset lies outside every 2-power subgroup in both CRT components), so the
// inverses come from one batch inversion.
__device__ __host__ inline qm31 composition(const QuotConsts& k, const qm31& x, const qm31* cur, const qm31* next,
                                            const qm31* pre, const qm31& zh, const qm31* per = nullptr,
                                            bool units = false) {
  qm31 res[kMaxTrans];
  if (per)
    rescue_stacked_eval(per, cur, next, res);
  else
    air_eval(k.air, x, cur, next, res);
  qm31 tsum = qzero();
  for (uint32_t t = 0; t < k.num_trans; ++t) tsum = qadd(tsum, qmul(k.alphas[t], res[t]));
  qm31 h = qmul(tsum, qsub(x, k.last_point));
  for (uint32_t r = 0; r < k.n_rel; ++r)
    h = qadd(h, qmul(k.alphas[k.num_trans + r], lookup_constraint(k, r, cur, pre, cur[k.m + r], next[k.m + r])));
  for (uint32_t r = 0; r < k.n_rel; ++r) {
    const qm31 sel = cur[k.sel[r]];
    h = qadd(h, qmul(k.alphas[k.num_trans + k.n_rel + r], qmul(sel, qsub(qone(), sel))));
  }
  if (k.total_bound == 0) return h;
  // acc_g = sum_{k: p_k = p_g} beta_k (f_k(x) - v_k), accumulated per group in a
  // register: local arrays written at run-time indices gave wrong results in this
  // kernel on the device, so the grouping is a comparison and the batch inversion keeps
  // no array of prefix products.
  qm31 bsum = qzero();
  if (units) {
    // 1 / (x - p_g) = prod_{h != g} (x - p_h) / prod_h (x - p_h): one inversion
    qm31 run = qone();
    for (uint32_t g = 0; g < k.n_bpts; ++g) run = qmul(run, qsub(x, k.bpts[g]));
    const qm31 inv = qinv(run);
    for (uint32_t g = 0; g < k.n_bpts; ++g) {
      qm31 ig = inv;
      for (uint32_t h2 = 0; h2 < k.n_bpts; ++h2)
        if (h2 != g) ig = qmul(ig, qsub(x, k.bpts[h2]));
      qm31 acc = qzero();
      for (uint32_t b = 0; b < k.total_bound; ++b)
        if (k.b_grp[b] == g) acc = qadd(acc, qmul(k.betas[b], qsub(cur[k.b_col[b]], k.b_val[b])));
      bsum = qadd(bsum, qmul(acc, ig));
    }
  } else {
    for (uint32_t g = 0; g < k.n_bpts; ++g) {
      qm31 acc = qzero();
      for (uint32_t b = 0; b < k.total_bound; ++b)
        if (k.b_grp[b] == g) acc = qadd(acc, qmul(k.betas[b], qsub(cur[k.b_col[b]], k.b_val[b])));
      bsum = qadd(bsum, qmul(acc, qinv(qsub(x, k.bpts[g]))));
    }
  }
  return qadd(h, qmul(bsum, zh));
}

}  // namespace zs
