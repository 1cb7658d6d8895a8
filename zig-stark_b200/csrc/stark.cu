// GenericStark(Air).proveWithPreprocessed (src/m31/stark.zig:327-658) on the device.
//
// The transcript (Channel) stays on the host and sees exactly the bytes the
// reference absorbs, in the same order; everything proportional to the trace or the
// domain runs on the GPU:
//   LDE of every column (QM31 NTT: interpolation on H, evaluation on D),
//   one Merkle tree per committed column (hashQM31 leaves),
//   the LogUp accumulator (row contributions + a parallel prefix sum),
//   the quotient Hc(x)/Z_H(x) on D,
//   the DEEP evaluations f_j(z), f_j(w z) (parallel Horner sums),
//   the DEEP codeword, the FRI layers (fold fused with the next layer's commitment),
//   and the gather of every revealed value and Merkle path.
// All device arithmetic is exact, so every root, layer and proof byte equals the
// reference's.
#include <algorithm>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "airs.cuh"
#include "constraints.cuh"
#include "fri.cuh"
#include "host.cuh"
#include "merkle.cuh"
#include "ntt.cuh"
#include "stark.cuh"
#include "staging.cuh"

namespace zs {

namespace {

constexpr unsigned kT = 256;

__device__ __forceinline__ qm31 ldq(const qm31* p) {
  const uint4 r = *reinterpret_cast<const uint4*>(p);
  return qmake(r.x, r.y, r.z, r.w);
}
__device__ __forceinline__ void stq(qm31* p, const qm31& v) {
  *reinterpret_cast<uint4*>(p) = make_uint4(v.a.a, v.a.b, v.b.a, v.b.b);
}

__device__ __forceinline__ qm31 domain_point(const QuotConsts& k, const qm31* __restrict__ wpow, uint32_t i) {
  // d_i = FRI_OFFSET * w_N^i, w_N^(N/2) = -1, wpow[k] = w_N^k for k < N/2
  const uint32_t half = 1u << (k.log_N - 1);
  qm31 w = i < half ? ldq(wpow + i) : qneg(ldq(wpow + (i - half)));
  return qmul(k.offset, w);
}

// The quotient's per-point tables: zh[2t] = Z_H(d_i), zh[2t + 1] = Z_H(d_i)^-1 for
// t = i mod 2^log_blowup (stark.zig:520-533 evaluates Z_H at every point; it takes only
// 2^log_blowup values on D), and for the stacked Rescue AIR the periodic values
// {y - w8^7, P_0(y), .., P_3(y)} of y = d_r^(n/8), which repeat with period 8 * 2^log_blowup.
__global__ void k_quot_tables(qm31* __restrict__ zh, qm31* __restrict__ per, const QuotConsts* __restrict__ kp,
                              qm31 wb, qm31 wN, uint32_t period) {
  const QuotConsts& k = *kp;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < (1u << k.log_blowup)) {
    const qm31 z = qsub(qmul(k.on, qpow(wb, t)), qone());
    stq(zh + 2 * (size_t)t, z);
    stq(zh + 2 * (size_t)t + 1, qinv(z));
  }
  if (per && t < period) {
    const qm31 y = qpow(qmul(k.offset, qpow(wN, t)), k.air.n_div8);
    qm31* row = per + (size_t)5 * t;
    stq(row, qsub(y, k.air.w8_7));
    for (int j = 0; j < 4; ++j) stq(row + 1 + j, horner(k.air.poly[j], 8, y));
  }
}

// cw: codewords of all columns ([pre | main | acc]), N each.
__global__ void __launch_bounds__(kT) k_quotient(const qm31* __restrict__ cw, qm31* __restrict__ q,
                                                 const qm31* __restrict__ wpow, const QuotConsts* __restrict__ kp,
                                                 const qm31* __restrict__ zh_tab, const qm31* __restrict__ per_tab) {
  const QuotConsts& k = *kp;
  const uint32_t N = 1u << k.log_N;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const uint32_t in = (i + k.shift) & (N - 1);
  qm31 cur[kMaxCols], next[kMaxCols], pre[kMaxPre];
  for (uint32_t j = 0; j < k.n_pre; ++j) pre[j] = ldq(cw + (size_t)j * N + i);
  for (uint32_t j = 0; j < k.m_total; ++j) {
    const qm31* c = cw + (size_t)(k.n_pre + j) * N;
    cur[j] = ldq(c + i);
    next[j] = ldq(c + in);
  }
  const qm31 x = domain_point(k, wpow, i);
  const uint32_t zi = i & ((1u << k.log_blowup) - 1);
  qm31 per[5];
  const bool stacked = k.air.id == AIR_RESCUE_STACKED;
  if (stacked)
    for (int j = 0; j < 5; ++j) per[j] = ldq(per_tab + (size_t)5 * (i & k.per_mask) + j);
  const qm31 h = composition(k, x, cur, next, pre, ldq(zh_tab + 2 * (size_t)zi), stacked ? per : nullptr, true);
  stq(q + i, qmul(h, ldq(zh_tab + 2 * (size_t)zi + 1)));
}

// The stacked Rescue AIR's quotient (12 columns, 12 transitions, boundaries on columns
// 0..3 at rows 0 and n - 1, no lookups) with every column index fixed at compile time, so
// the row stays in registers (the generic kernel's run-time indices put its column
// arrays in local memory). The boundary sum is taken per point p_g as
// sum_j c_gj f_j(x) - e_g, with c_gj = sum_{b: p_b = p_g, col_b = j} beta_b and
// e_g = sum_{b: p_b = p_g} beta_b v_b formed on the host: equal in the field to the
// generic sum_b beta_b (f_col_b(x) - v_b), term by term.
struct RescueQuot {
  qm31 alphas[12];
  qm31 bc[2][4];  // c_gj
  qm31 be[2];     // e_g
  qm31 bp[2];     // p_g
};

__global__ void __launch_bounds__(kT) k_quotient_rescue(const qm31* __restrict__ cw, qm31* __restrict__ q,
                                                        const qm31* __restrict__ wpow,
                                                        const QuotConsts* __restrict__ kp,
                                                        const __grid_constant__ RescueQuot rq,
                                                        const qm31* __restrict__ zh_tab,
                                                        const qm31* __restrict__ per_tab) {
  const QuotConsts& k = *kp;
  const uint32_t N = 1u << k.log_N;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const uint32_t in = (i + k.shift) & (N - 1);
  qm31 cur[12], next[4], per[5], res[12];
#pragma unroll
  for (int j = 0; j < 12; ++j) cur[j] = ldq(cw + (size_t)j * N + i);
#pragma unroll
  for (int j = 0; j < 4; ++j) next[j] = ldq(cw + (size_t)j * N + in);
#pragma unroll
  for (int j = 0; j < 5; ++j) per[j] = ldq(per_tab + (size_t)5 * (i & k.per_mask) + j);
  const qm31 x = domain_point(k, wpow, i);
  rescue_stacked_eval(per, cur, next, res);
  qm31 tsum = qzero();
#pragma unroll
  for (int t = 0; t < 12; ++t) tsum = qadd(tsum, qmul(rq.alphas[t], res[t]));
  qm31 h = qmul(tsum, qsub(x, k.last_point));
  const qm31 d0 = qsub(x, rq.bp[0]), d1 = qsub(x, rq.bp[1]);
  const qm31 inv = qinv(qmul(d0, d1));  // every x - p is a unit on the evaluation domain
  qm31 acc0 = qneg(rq.be[0]), acc1 = qneg(rq.be[1]);
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    acc0 = qadd(acc0, qmul(rq.bc[0][j], cur[j]));
    acc1 = qadd(acc1, qmul(rq.bc[1][j], cur[j]));
  }
  const qm31 bsum = qadd(qmul(acc0, qmul(inv, d1)), qmul(acc1, qmul(inv, d0)));
  const uint32_t zi = i & ((1u << k.log_blowup) - 1);
  h = qadd(h, qmul(bsum, ldq(zh_tab + 2 * (size_t)zi)));
  stq(q + i, qmul(h, ldq(zh_tab + 2 * (size_t)zi + 1)));
}

// The RescueQuot of `k`, when its constraints have the stacked Rescue shape the
// specialised kernel assumes (checked, not assumed).
bool rescue_quot(const QuotConsts& k, RescueQuot& rq) {
  if (k.air.id != AIR_RESCUE_STACKED || k.m != 12 || k.m_total != 12 || k.num_trans != 12 || k.n_rel != 0 ||
      k.n_pre != 0 || k.n_bpts != 2)
    return false;
  for (int t = 0; t < 12; ++t) rq.alphas[t] = k.alphas[t];
  for (int g = 0; g < 2; ++g) {
    rq.bp[g] = k.bpts[g];
    rq.be[g] = qzero();
    for (int j = 0; j < 4; ++j) rq.bc[g][j] = qzero();
  }
  for (uint32_t b = 0; b < k.total_bound; ++b) {
    const uint32_t g = k.b_grp[b], j = k.b_col[b];
    if (g >= 2 || j >= 4) return false;
    rq.bc[g][j] = qadd(rq.bc[g][j], k.betas[b]);
    rq.be[g] = qadd(rq.be[g], qmul(k.betas[b], k.b_val[b]));
  }
  return true;
}

// LogUp row contributions (stark.zig:283-297) on H: out[i] = contribution of row i.
__global__ void k_logup_rows(const qm31* __restrict__ vals, uint32_t n, const QuotConsts* __restrict__ kp,
                             uint32_t r, qm31* __restrict__ out) {
  const QuotConsts& k = *kp;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  qm31 row[kMaxCols], pre[kMaxPre];
  for (uint32_t j = 0; j < k.n_pre; ++j) pre[j] = ldq(vals + (size_t)j * n + i);
  for (uint32_t j = 0; j < k.m; ++j) row[j] = ldq(vals + (size_t)(k.n_pre + j) * n + i);
  const qm31 sel = row[k.sel[r]], mult = row[k.mult[r]];
  const qm31 key = combined_key(k.ac, k.n_keys[r], k.keys[r], row);
  const qm31 tkey = combined_key(k.ac, k.n_keys[r], k.tabs[r], pre);
  const qm31 lt = qmul(sel, qmul(mult, qinv(qsub(k.ar[r], key))));
  const qm31 tt = qmul(qsub(qone(), sel), qinv(qsub(k.ar[r], tkey)));
  stq(out + i, qsub(lt, tt));
}

// The linear-layer AIR's LogUp row contributions (stark.zig:283-297) on H, its key and
// table columns streamed from the column-major values [P_0..P_127 | x, y, sel, mult].
__global__ void __launch_bounds__(kT) k_ml_logup_rows(const qm31* __restrict__ vals, uint32_t n,
                                                      const MlConsts* __restrict__ kp, qm31* __restrict__ out) {
  const MlConsts& k = *kp;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const qm31* main = vals + (size_t)kMlDim * n;
  qm31 key = qzero(), tkey = qzero();
  for (uint32_t l = 0; l < kMlDim; ++l) {
    key = qadd(key, qmul(k.ac[l], ldq(main + (size_t)l * n + i)));
    tkey = qadd(tkey, qmul(k.ac[l], ldq(vals + (size_t)l * n + i)));
  }
  const qm31 sel = ldq(main + (size_t)kMlSel * n + i), mult = ldq(main + (size_t)kMlMult * n + i);
  const qm31 lt = qmul(sel, qmul(mult, qinv(qsub(k.ar, key))));
  const qm31 tt = qmul(qsub(qone(), sel), qinv(qsub(k.ar, tkey)));
  stq(out + i, qsub(lt, tt));
}

// The linear-layer AIR's quotient Hc(d_i) / Z_H(d_i) on D: ml_composition
// (constraints.cuh) with the row's 387 values streamed from the codewords
// [P_0..P_127 | x, y, sel, mult | acc] instead of held per thread.
__global__ void __launch_bounds__(kT) k_ml_quotient(const qm31* __restrict__ cw, qm31* __restrict__ q,
                                                    const qm31* __restrict__ wpow, const MlConsts* __restrict__ kp,
                                                    const qm31* __restrict__ zh_tab) {
  const MlConsts& k = *kp;
  const uint32_t N = 1u << k.log_N;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const uint32_t half = N >> 1;
  const qm31 x = qmul(k.offset, i < half ? ldq(wpow + i) : qneg(ldq(wpow + (i - half))));
  const qm31* main = cw + (size_t)kMlDim * N;
  qm31 ty = qzero(), tx = qzero(), key = qzero(), tkey = qzero();
  for (uint32_t l = 0; l < kMlDim; ++l) {
    const qm31 xl = ldq(main + (size_t)l * N + i);
    ty = qadd(ty, qmul(k.alpha_y[l], ldq(main + (size_t)(kMlDim + l) * N + i)));
    tx = qadd(tx, qmul(k.beta_x[l], xl));
    key = qadd(key, qmul(k.ac[l], xl));
    tkey = qadd(tkey, qmul(k.ac[l], ldq(cw + (size_t)l * N + i)));
  }
  const uint32_t in = (i + k.shift) & (N - 1);
  const qm31 sel = ldq(main + (size_t)kMlSel * N + i), mult = ldq(main + (size_t)kMlMult * N + i);
  const qm31 acc = ldq(main + (size_t)kMlCols * N + i), accn = ldq(main + (size_t)kMlCols * N + in);
  qm31 h = qmul(qsub(ty, tx), qsub(x, k.last_point));
  const qm31 dacc = qsub(accn, acc);
  const qm31 lb = qsub(qmul(dacc, qsub(k.ar, key)), mult);
  const qm31 tb = qadd(qmul(dacc, qsub(k.ar, tkey)), qone());
  h = qadd(h, qmul(k.alpha_look, qadd(qmul(sel, lb), qmul(qsub(qone(), sel), tb))));
  h = qadd(h, qmul(k.alpha_bin, qmul(sel, qsub(qone(), sel))));
  const qm31 d_sel = qsub(x, k.last_point), d_acc = qsub(x, qone());
  const qm31 inv = qinv(qmul(d_sel, d_acc));
  const qm31 b = qadd(qmul(k.beta_sel, qmul(sel, qmul(inv, d_acc))), qmul(k.beta_acc, qmul(acc, qmul(inv, d_sel))));
  const uint32_t zi = i & ((1u << k.log_blowup) - 1);
  h = qadd(h, qmul(b, ldq(zh_tab + 2 * (size_t)zi)));
  stq(q + i, qmul(h, ldq(zh_tab + 2 * (size_t)zi + 1)));
}

// Exclusive prefix sum of QM31 values in blocks of 1024 (exact, so any association
// order gives the reference's acc[i] = sum_{k<i} c_k).
__global__ void __launch_bounds__(1024) k_scan_block(const qm31* in, qm31* out, uint32_t n, qm31* block_sums) {
  __shared__ qm31 s[1024];
  const uint32_t i = blockIdx.x * 1024 + threadIdx.x;
  s[threadIdx.x] = i < n ? ldq(in + i) : qzero();
  __syncthreads();
  for (uint32_t d = 1; d < 1024; d <<= 1) {
    qm31 v = threadIdx.x >= d ? s[threadIdx.x - d] : qzero();
    __syncthreads();
    s[threadIdx.x] = qadd(s[threadIdx.x], v);
    __syncthreads();
  }
  // inclusive in s; exclusive output
  if (i < n) stq(out + i, threadIdx.x == 0 ? qzero() : s[threadIdx.x - 1]);
  if (threadIdx.x == 1023 && block_sums) stq(block_sums + blockIdx.x, s[1023]);
}

__global__ void k_scan_add(qm31* out, uint32_t n, const qm31* block_prefix) {
  const uint32_t i = blockIdx.x * 1024 + threadIdx.x;
  if (i < n && blockIdx.x > 0) stq(out + i, qadd(ldq(out + i), ldq(block_prefix + blockIdx.x)));
}

// A block's kT threads sum kT * kEvalPer terms; QM31 addition is exact, so the order
// of the sums does not change the result.
constexpr uint32_t kEvalPer = 8;

__device__ __forceinline__ qm31 block_sum(qm31 v, qm31* s) {
  s[threadIdx.x] = v;
  __syncthreads();
  for (uint32_t d = blockDim.x / 2; d > 0; d >>= 1) {
    if (threadIdx.x < d) s[threadIdx.x] = qadd(s[threadIdx.x], s[threadIdx.x + d]);
    __syncthreads();
  }
  return s[0];
}

// partial[pt][col][blk] = sum over the block's j of coeffs[col][j] * zpow[pt][bitrev(j)]
// (the coefficients are stored in bit-reversed order, log_n = log2 n).
__global__ void __launch_bounds__(kT) k_eval_partial(const qm31* __restrict__ coeffs, uint32_t n, unsigned log_n,
                                                     const qm31* __restrict__ zpow, uint32_t npt, qm31* partial) {
  __shared__ qm31 s[kT];
  const uint32_t col = blockIdx.y, pt = blockIdx.z;
  const qm31* c = coeffs + (size_t)col * n;
  const qm31* zp = zpow + (size_t)pt * n;
  qm31 acc = qzero();
#pragma unroll
  for (uint32_t k = 0; k < kEvalPer; ++k) {
    const uint32_t j = (blockIdx.x * kEvalPer + k) * blockDim.x + threadIdx.x;
    if (j < n) acc = qadd(acc, qmul(ldq(c + j), ldq(zp + bitrev(j, log_n))));
  }
  const qm31 sum = block_sum(acc, s);
  if (threadIdx.x == 0) stq(partial + ((size_t)pt * gridDim.y + col) * gridDim.x + blockIdx.x, sum);
}

// out[idx] = the sum of the `nblk` partials of (pt, col) = idx, one CTA each.
__global__ void __launch_bounds__(kT) k_eval_sum(const qm31* partial, uint32_t nblk, qm31* out) {
  __shared__ qm31 s[kT];
  const qm31* p = partial + (size_t)blockIdx.x * nblk;
  qm31 acc = qzero();
  for (uint32_t b = threadIdx.x; b < nblk; b += blockDim.x) acc = qadd(acc, ldq(p + b));
  const qm31 sum = block_sum(acc, s);
  if (threadIdx.x == 0) stq(out + blockIdx.x, sum);
}

// DEEP codeword (stark.zig:577-588), with 1/(d_i - z) factored out of the sum.
// ge: the 2 m_total + 1 weights gamma_j, then the 2 m_total evaluations f_j(z), f_j(wz).
struct DeepConsts {
  uint32_t m_total, n_pre, shift;
  unsigned log_N;
  qm31 offset, z, qz;
};

__global__ void __launch_bounds__(kT) k_deep(const qm31* __restrict__ cw, const qm31* __restrict__ q,
                                             const qm31* __restrict__ wpow, const DeepConsts* __restrict__ kp,
                                             const qm31* __restrict__ ge, qm31* __restrict__ g) {
  const DeepConsts& k = *kp;
  const qm31* gammas = ge;
  const qm31* evals = ge + 2 * k.m_total + 1;
  const uint32_t N = 1u << k.log_N;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const uint32_t in = (i + k.shift) & (N - 1);
  const uint32_t half = N >> 1;
  const qm31 w = i < half ? ldq(wpow + i) : qneg(ldq(wpow + (i - half)));
  const qm31 x = qmul(k.offset, w);
  const qm31 inv_dz = qinv(qsub(x, k.z));
  qm31 acc = qzero();
  for (uint32_t j = 0; j < k.m_total; ++j) {
    const qm31* c = cw + (size_t)(k.n_pre + j) * N;
    acc = qadd(acc, qmul(ldq(gammas + j), qsub(ldq(c + i), ldq(evals + j))));
    acc = qadd(acc, qmul(ldq(gammas + k.m_total + j), qsub(ldq(c + in), ldq(evals + k.m_total + j))));
  }
  acc = qadd(acc, qmul(ldq(gammas + 2 * k.m_total), qsub(ldq(q + i), k.qz)));
  stq(g + i, qmul(acc, inv_dz));
}

// Gather: out[r] = words [idx * w, (idx + 1) * w) of src[r] (requests prepared on the host).
// One entry of a query's gather list: `words` words (4: a QM31 value, 8: a Merkle node)
// from `base` at element index idx, where the query's position p is p0 mod 2^modlog
// (kQLow), that plus 2^modlog (kQHigh), p0 itself (kQP0) or (p0 + shift) mod 2^lN
// (kQShift), and idx = p for a value or (p >> lvl) ^ 1, the sibling at level lvl, for a
// path node. `off` is its word offset within the query's slice of section `sec`.
enum : uint8_t { kQLow = 0, kQHigh = 1, kQP0 = 2, kQShift = 3 };
constexpr uint8_t kQValue = 0xff;
struct QueryReq {
  const uint32_t* base;
  uint32_t off;
  uint16_t words;
  uint8_t sec, mode, modlog, lvl;
};
// One FRI transcript step on the device (fri.zig:199-206): absorb the layer root,
// sample the folding challenge. One warp copies the state to shared memory and back;
// one thread runs the step there.
__global__ void k_fri_transcript(Channel* ch, const uint32_t* __restrict__ root, uint32_t* __restrict__ root_out,
                                 qm31* __restrict__ alpha) {
  __shared__ __align__(16) unsigned char ch_raw[sizeof(Channel)];
  copy_state(ch_raw, ch, sizeof(Channel));
  __syncthreads();
  if (threadIdx.x == 0) {
    Channel* c = reinterpret_cast<Channel*>(ch_raw);
    uint8_t b[32];
    for (int w = 0; w < 8; ++w) {
      const uint32_t v = root[w];
      root_out[w] = v;
      for (int k = 0; k < 4; ++k) b[4 * w + k] = (uint8_t)(v >> (8 * k));
    }
    c->absorb_bytes(b, 32);
    *alpha = c->sample_q();
  }
  __syncthreads();
  copy_state(ch, ch_raw, sizeof(Channel));
}

// The gathered words of every query: query qi's section-0 words at qi * sec0, its
// section-1 words after all nq queries' section 0, at nq * sec0 + qi * sec1. Grid:
// (entries of the template, queries q0 .. q0 + gridDim.y - 1).
__global__ void k_gather_queries(const QueryReq* __restrict__ tmpl, uint32_t count, const uint64_t* __restrict__ p0s,
                                 uint32_t q0, uint32_t nq, uint64_t shift, unsigned log_N, uint32_t sec0,
                                 uint32_t sec1, uint32_t* __restrict__ out) {
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x, qi = q0 + blockIdx.y;
  if (e >= count) return;
  const QueryReq r = tmpl[e];
  const uint64_t p0 = p0s[qi], low = p0 & (((uint64_t)1 << r.modlog) - 1);
  uint64_t p = p0;
  if (r.mode == kQLow) p = low;
  else if (r.mode == kQHigh) p = low + ((uint64_t)1 << r.modlog);
  else if (r.mode == kQShift) p = (p0 + shift) & (((uint64_t)1 << log_N) - 1);
  const uint64_t idx = r.lvl == kQValue ? p : ((p >> r.lvl) ^ 1);
  uint32_t* dst = out + (r.sec == 0 ? (size_t)qi * sec0 : (size_t)nq * sec0 + (size_t)qi * sec1) + r.off;
  for (uint32_t w = 0; w < r.words; ++w) dst[w] = r.base[idx * r.words + w];
}

template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaStream_t st = nullptr;
  DevBuf() = default;
  DevBuf(size_t count, cudaStream_t s) : n(count), st(s) {
    ZS_CUDA(cudaMallocAsync((void**)&p, (count ? count : 1) * sizeof(T), s));
  }
  ~DevBuf() {
    if (p) cudaFreeAsync(p, st);
  }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
};

Digest root_of(const DeviceTree& t, cudaStream_t st) {
  Digest d;
  d2h_small(d.data(), t.root(), 32, st);
  return d;
}

struct OwnedTree {
  DeviceTree t;
  cudaStream_t st;
  OwnedTree(unsigned log_n, cudaStream_t s) : st(s) {
    t.log_n = log_n;
    ZS_CUDA(cudaMallocAsync((void**)&t.words, DeviceTree::words_for(log_n) * sizeof(uint32_t), s));
  }
  ~OwnedTree() { cudaFreeAsync(t.words, st); }
};

// Size-only tables (NTT twiddles, powers of FRI_OFFSET, fold tables) of sizes up to
// 2^kCacheLog are built once per device and shared by every later proof: the first
// use builds them on a private stream and waits for it, after which they are
// read-only and visible to every stream. The cache is never freed (it would outlive
// the CUDA context at process exit). Larger tables are built per proof on its stream.
constexpr unsigned kCacheLog = 20;

template <typename T, typename Make>
const T& cached_table(unsigned log_n, Make&& make) {
  static std::mutex mu;
  static auto* cache = new std::map<std::pair<int, unsigned>, T*>();
  int dev = 0;
  ZS_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache->find({dev, log_n});
  if (it != cache->end()) return *it->second;
  cudaStream_t s = nullptr;
  ZS_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  T* t = nullptr;
  try {
    t = make(s);
    ZS_CUDA(cudaStreamSynchronize(s));
  } catch (...) {
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    throw;
  }
  cudaStreamDestroy(s);
  (*cache)[{dev, log_n}] = t;
  return *t;
}

const NttTables& ntt_tables(unsigned log_n, cudaStream_t st, std::unique_ptr<NttTables>& own) {
  if (log_n > kCacheLog) {
    own = std::make_unique<NttTables>(log_n, st);
    return *own;
  }
  return cached_table<NttTables>(log_n, [&](cudaStream_t s) { return new NttTables(log_n, s); });
}

const FoldTables& fold_tables(unsigned dlog, cudaStream_t st, std::unique_ptr<FoldTables>& own) {
  if (dlog > kCacheLog) {
    own = std::make_unique<FoldTables>(dlog, st);
    return *own;
  }
  return cached_table<FoldTables>(dlog, [&](cudaStream_t s) { return new FoldTables(dlog, s); });
}

// FRI_OFFSET^k for k < 2^log_n.
struct OffsetPowers {
  qm31* p = nullptr;
  OffsetPowers(unsigned log_n, cudaStream_t s) {
    ZS_CUDA(cudaMallocAsync(&p, sizeof(qm31) << log_n, s));
    qm31_powers(q_fri_offset(), p, 1u << log_n, s);
  }
};
const qm31* offset_powers(unsigned log_n, cudaStream_t st, std::unique_ptr<DevBuf<qm31>>& own) {
  if (log_n > kCacheLog) {
    own = std::make_unique<DevBuf<qm31>>((size_t)1 << log_n, st);
    qm31_powers(q_fri_offset(), own->p, 1u << log_n, st);
    return own->p;
  }
  return cached_table<OffsetPowers>(log_n, [&](cudaStream_t s) { return new OffsetPowers(log_n, s); }).p;
}

// The roots of trees[a, b), read back with one wait.
std::vector<Digest> roots_of(const std::vector<std::unique_ptr<OwnedTree>>& trees, uint32_t a, uint32_t b,
                             cudaStream_t st) {
  std::vector<Digest> out(b - a);
  std::vector<D2H> c;
  for (uint32_t j = a; j < b; ++j) c.push_back({out[j - a].data(), trees[j]->t.root(), 32});
  d2h_many(c.data(), c.size(), st);
  return out;
}

// The DeviceTree pointers of trees[a, b).
std::vector<DeviceTree*> tree_ptrs(const std::vector<std::unique_ptr<OwnedTree>>& trees, uint32_t a, uint32_t b) {
  std::vector<DeviceTree*> v;
  for (uint32_t j = a; j < b; ++j) v.push_back(&trees[j]->t);
  return v;
}

// The columns of a wire []const []const QM31, located but not decoded: each element
// is four little-endian u32 words, the device layout of a qm31, so a column's bytes
// go to the device as they are and M31.fromBytes' reduction (m31.zig:97-100) runs
// there (k_from_bytes).
struct WireColumns {
  std::vector<const uint8_t*> data;
  std::vector<uint64_t> len;
  size_t size() const { return data.size(); }
};

WireColumns locate_columns(const uint8_t* d, size_t n) {
  WireColumns c;
  if (n == 0) return c;
  WireReader r(d, n);
  const uint64_t m = r.len(8);
  for (uint64_t j = 0; j < m; ++j) {
    const uint64_t len = r.len(16);
    c.data.push_back(r.take(16 * len));
    c.len.push_back(len);
  }
  r.end();
  return c;
}

// Column data of the wire span -> canonical M31 words. Column j's element words
// start 2 + 4n words after column j-1's (its u64 length prefix sits between them);
// raw < 2^32 <= 2p + 2, so at most two subtractions reduce it.
__global__ void k_from_wire(const uint32_t* __restrict__ raw, uint32_t* __restrict__ out, uint64_t col_words,
                            uint64_t count) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const uint64_t j = i / col_words;
  uint32_t v = raw[i + 2 * j];
  v = v >= P ? v - P : v;
  v = v >= P ? v - P : v;
  out[i] = v;
}

// wire words of an M31 -> canonical QM31 (v, 0, 0, 0); raw < 2^32 <= 2p + 2
__global__ void k_from_low(const uint32_t* __restrict__ low, qm31* __restrict__ out, uint64_t count) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  uint32_t v = low[i];
  v = v >= P ? v - P : v;
  v = v >= P ? v - P : v;
  reinterpret_cast<uint4*>(out)[i] = make_uint4(v, 0, 0, 0);
}

// Copies the columns of `c` (each of n elements) to dst (column k at dst + k * n) and
// reduces them. Large traces cross PCIe packed: the low word of every element, with the
// columns whose upper words are not all zero (true QM31 values) uploaded again whole.
// Small ones go as the span of the caller's buffer that holds all columns in one upload,
// and a kernel drops the length prefixes between the columns.
constexpr size_t kPackMin = (size_t)4 << 20;  // wire bytes from which packing pays
void upload_columns(const WireColumns& c, qm31* dst, uint32_t n, cudaStream_t st) {
  if (c.size() == 0) return;
  const uint32_t C = (uint32_t)c.size();
  const uint64_t col_words = (uint64_t)4 * n, count = col_words * C;
  const size_t span = (size_t)(c.data.back() - c.data.front()) + (size_t)16 * n;
  if (span >= kPackMin) {
    DevBuf<uint32_t> low((size_t)C * n, st);
    std::vector<uint8_t> high(C);
    upload_low_words(low.p, c.data.data(), C, n, high.data(), st);
    const uint64_t elems = (uint64_t)C * n;
    k_from_low<<<(unsigned)((elems + 255) / 256), 256, 0, st>>>(low.p, dst, elems);
    ZS_CUDA(cudaGetLastError());
    for (uint32_t j = 0; j < C; ++j) {
      if (!high[j]) continue;
      DevBuf<uint32_t> raw(col_words, st);
      upload_bytes(raw.p, c.data[j], (size_t)16 * n, st);
      k_from_wire<<<(unsigned)((col_words + 255) / 256), 256, 0, st>>>(raw.p, reinterpret_cast<uint32_t*>(dst + (size_t)j * n),
                                                                       col_words, col_words);
      ZS_CUDA(cudaGetLastError());
    }
    return;
  }
  DevBuf<uint32_t> raw((span + 3) / 4, st);
  upload_bytes(raw.p, c.data.front(), span, st);
  k_from_wire<<<(unsigned)((count + 255) / 256), 256, 0, st>>>(raw.p, reinterpret_cast<uint32_t*>(dst), col_words,
                                                              count);
  ZS_CUDA(cudaGetLastError());
}

// A side stream for one proof's uploads or trees (the calling thread's stream in `slot`),
// forked from `st` (so it sees the buffers allocated there before). join() makes `st`
// wait for everything issued on it so far; the destructor joins too (so stream-ordered
// frees on `st` follow every copy) and waits for the side stream to drain.
struct CopyStream {
  cudaStream_t s = nullptr, st;
  cudaEvent_t ev = nullptr;
  CopyStream(cudaStream_t main, int slot) : st(main) {
    thread_stream(slot, &s, &ev);
    fork();  // buffers allocated on `st` so far are ready
  }
  void join() {
    ZS_CUDA(cudaEventRecord(ev, s));
    ZS_CUDA(cudaStreamWaitEvent(st, ev, 0));
  }
  void fork() {  // the side stream waits for everything issued on `st` so far
    ZS_CUDA(cudaEventRecord(ev, st));
    ZS_CUDA(cudaStreamWaitEvent(s, ev, 0));
  }
  ~CopyStream() {
    cudaEventRecord(ev, s);
    cudaStreamWaitEvent(st, ev, 0);
    cudaStreamSynchronize(s);
  }
  CopyStream(const CopyStream&) = delete;
  CopyStream& operator=(const CopyStream&) = delete;
};
constexpr size_t kPriorityUpload = (size_t)64 << 20;  // wire bytes from which uploads wait for the copy pool
constexpr size_t kGroupMin = (size_t)8 << 20;    // wire bytes below which one group suffices
constexpr size_t kGroupBytes = (size_t)16 << 20;  // wire bytes per upload group

}  // namespace

std::vector<uint8_t> stark_prove(uint32_t air_id, const uint8_t* params_b, size_t params_len, const uint8_t* pi,
                                 size_t pi_len, const uint8_t* pre_b, size_t pre_len, const uint8_t* trace_b,
                                 size_t trace_len, const uint8_t* sep, size_t sep_len, cudaStream_t st) {
  // ---- inputs -------------------------------------------------------------
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
  const WireColumns pre = locate_columns(pre_b, pre_len);
  const WireColumns trace = locate_columns(trace_b, trace_len);
  const unsigned tl = sp.trace_log, lb = sp.log_blowup, lN = tl + lb;
  if (lN > 26) throw Error(ZS_EMALFORMED, "trace_log + log_blowup above 26");
  if (sp.num_queries > ((uint64_t)1 << 24)) throw Error(ZS_EMALFORMED, "more than 2^24 queries");
  const uint32_t n = 1u << tl, N = 1u << lN, shift = 1u << lb;
  if (air.fixed_n && n != air.fixed_n) throw Error(ZS_EMALFORMED, "the AIR is defined for a fixed trace length");
  if (air.id == AIR_RESCUE_STACKED && n < 8) throw Error(ZS_EMALFORMED, "stacked rescue needs at least 8 rows");
  if (trace.size() != air.m || pre.size() != air.n_pre) throw Error(ZS_EMALFORMED, "column count mismatch");
  retain_pool_memory();
  PinnedScope pinned(st);
  UploadPriority upload_priority(trace_len + pre_len >= kPriorityUpload);
  for (uint64_t l : trace.len)
    if (l != n) throw Error(ZS_EMALFORMED, "column length mismatch");
  for (uint64_t l : pre.len)
    if (l != n) throw Error(ZS_EMALFORMED, "column length mismatch");
  const uint32_t m = air.m, n_pre = air.n_pre, n_rel = air.n_rel, m_total = m + n_rel;
  const uint32_t n_trans_total = air.num_trans + 2 * n_rel, total_bound = air.num_bound + n_rel;
  const uint32_t n_deep = 2 * m_total + 1, reveal_len = 2 * m_total + 1 + n_pre;
  const bool wide = air.id == AIR_ML_LINEAR;  // streamed by its own kernels
  if (!wide && (m_total > kMaxCols || air.num_trans > kMaxTrans || total_bound > kMaxBound || n_pre > kMaxPre))
    throw Error(ZS_EGENERIC, "AIR exceeds the compiled-in limits");
  // FRI parameters (stark.zig:197-239)
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
    if (fp.remainder_log < fp.log_blowup) throw Error(ZS_EPROTOCOL, "remainder_log below the FRI blowup");
  }
  const unsigned L = fp.folds();
  const qm31 w = q_root_of_unity(tl), offset = q_fri_offset();

  // ---- LDE of preprocessed and main columns ------------------------------------
  const uint32_t ncol = n_pre + m_total;  // [pre | main | acc]
  std::unique_ptr<NttTables> small_own, big_own;
  std::unique_ptr<DevBuf<qm31>> pows_own;
  const NttTables& small = ntt_tables(tl, st, small_own);
  const NttTables& big = ntt_tables(lN, st, big_own);
  const qm31* offset_pows = offset_powers(tl, st, pows_own);
  DevBuf<qm31> vals((size_t)ncol * n, st), coeffs((size_t)ncol * n, st), cw((size_t)ncol * N, st);
  std::vector<std::unique_ptr<OwnedTree>> trees;
  for (uint32_t j = 0; j < ncol; ++j) trees.push_back(std::make_unique<OwnedTree>(lN, st));
  {
    // Columns [pre | main] in groups: group g+1 is packed on the host and copied on a
    // copy stream while the LDE of group g runs on `st` and its trees on a side stream
    // (so the narrow, latency-bound top levels of one group's trees overlap the next
    // group's transforms). Group sizes double from one column up to kGroupBytes: the
    // device starts after one column's packing, and since it spends about twice as long
    // on a column as the host spends packing one, each group is packed before the device
    // finishes the one before it. A proof whose columns are small goes as one group.
    const uint32_t C = n_pre + m;
    const size_t col_bytes = (size_t)16 * n;
    const uint32_t per = col_bytes * C < kGroupMin ? C : std::max<uint32_t>(1, (uint32_t)(kGroupBytes / col_bytes));
    std::unique_ptr<CopyStream> cs, ts;
    if (per < C) cs = std::make_unique<CopyStream>(st, 1), ts = std::make_unique<CopyStream>(st, 2);
    cudaStream_t up = cs ? cs->s : st;
    uint32_t gsize = per < C ? 1 : per;
    for (uint32_t c0 = 0; c0 < C;) {
      const uint32_t c1 = std::min(C, c0 + gsize);
      gsize = std::min(per, 2 * gsize);
      WireColumns gp, gt;  // this group's preprocessed and main columns
      for (uint32_t j = c0; j < std::min(c1, n_pre); ++j) gp.data.push_back(pre.data[j]), gp.len.push_back(n);
      for (uint32_t j = std::max(c0, n_pre); j < c1; ++j)
        gt.data.push_back(trace.data[j - n_pre]), gt.len.push_back(n);
      upload_columns(gp, vals.p + (size_t)c0 * n, n, up);
      upload_columns(gt, vals.p + (size_t)std::max(c0, n_pre) * n, n, up);
      if (cs) cs->join();  // `st` waits for this group's columns only
      lde_qm31(vals.p + (size_t)c0 * n, n, coeffs.p + (size_t)c0 * n, n, cw.p + (size_t)c0 * N, N, c1 - c0, small,
               big, offset_pows, st);
      if (ts) {
        ts->fork();
        build_qm31_trees(cw.p + (size_t)c0 * N, N, tree_ptrs(trees, c0, c1).data(), c1 - c0, ts->s);
      } else {
        build_qm31_trees(cw.p + (size_t)c0 * N, N, tree_ptrs(trees, c0, c1).data(), c1 - c0, st);
      }
      c0 = c1;
    }
    if (ts) ts->join();  // the roots below are read on `st`
  }

  Channel ch(sep, sep_len);
  WireWriter proof;
  proof.u8(sp.trace_log);
  proof.u8(sp.log_blowup);
  proof.u64(sp.num_queries);
  proof.u8(sp.remainder_log);
  std::vector<Digest> pre_roots, trace_roots, acc_roots;
  {
    const std::vector<Digest> roots = roots_of(trees, 0, n_pre + m, st);
    pre_roots.assign(roots.begin(), roots.begin() + n_pre);
    trace_roots.assign(roots.begin() + n_pre, roots.end());
  }
  for (const Digest& d : pre_roots) ch.absorb(d);
  for (const Digest& d : trace_roots) ch.absorb(d);

  // ---- LogUp challenges and accumulators ---------------------------------------
  QuotConsts kc{};
  kc.air = air.consts;
  kc.air.n_div8 = n / 8;
  kc.m = m, kc.m_total = m_total, kc.n_pre = n_pre, kc.num_trans = air.num_trans, kc.n_rel = n_rel;
  kc.total_bound = total_bound, kc.shift = shift, kc.log_N = lN, kc.log_blowup = lb;
  kc.offset = offset;
  kc.last_point = qpow(w, n - 1);
  std::vector<qm31> ac(air.n_lc), ar(n_rel);
  for (auto& a : ac) a = ch.sample_q();
  for (auto& a : ar) a = ch.sample_q();
  DevBuf<QuotConsts> d_kc(1, st);
  std::unique_ptr<MlConsts> ml;
  std::unique_ptr<DevBuf<MlConsts>> d_ml;
  if (wide) {
    ml = std::make_unique<MlConsts>();
    for (uint32_t l = 0; l < kMlDim; ++l) ml->ac[l] = ac[l];
    ml->ar = ar[0];
    ml->last_point = kc.last_point, ml->offset = offset;
    ml->log_N = lN, ml->log_blowup = lb, ml->shift = shift;
    d_ml = std::make_unique<DevBuf<MlConsts>>(1, st);
    h2d_small(d_ml->p, ml.get(), sizeof(MlConsts), st);
  } else {
    for (uint32_t j = 0; j < air.n_lc; ++j) kc.ac[j] = ac[j];
    for (uint32_t r = 0; r < n_rel; ++r) kc.ar[r] = ar[r];
    for (uint32_t r = 0; r < n_rel; ++r) {
      kc.sel[r] = air.sel[r], kc.mult[r] = air.mult[r], kc.n_keys[r] = air.n_keys[r];
      for (uint32_t j = 0; j < air.n_keys[r]; ++j) kc.keys[r][j] = air.keys[r][j], kc.tabs[r][j] = air.tabs[r][j];
    }
    if (const char* bad = quot_consts_out_of_range(kc, shift, true)) throw Error(ZS_EGENERIC, bad);
    h2d_small(d_kc.p, &kc, sizeof(kc), st);
  }
  if (n_rel > 0) {
    DevBuf<qm31> contrib(n, st);
    const uint32_t nb = (n + 1023) / 1024;
    DevBuf<qm31> sums(nb, st), sums_scan(nb, st);
    for (uint32_t r = 0; r < n_rel; ++r) {
      qm31* acc_vals = vals.p + (size_t)(n_pre + m + r) * n;
      if (wide)
        k_ml_logup_rows<<<(n + kT - 1) / kT, kT, 0, st>>>(vals.p, n, d_ml->p, contrib.p);
      else
        k_logup_rows<<<(n + kT - 1) / kT, kT, 0, st>>>(vals.p, n, d_kc.p, r, contrib.p);
      // acc[i] = sum_{k < i} contrib[k] (stark.zig:438-446)
      k_scan_block<<<nb, 1024, 0, st>>>(contrib.p, acc_vals, n, sums.p);
      if (nb > 1) {
        if (nb > 1024) throw Error(ZS_EGENERIC, "trace too long for the accumulator scan");
        k_scan_block<<<1, 1024, 0, st>>>(sums.p, sums_scan.p, nb, nullptr);
        k_scan_add<<<nb, 1024, 0, st>>>(acc_vals, n, sums_scan.p);
      }
    }
    ZS_CUDA(cudaGetLastError());
    lde_qm31(vals.p + (size_t)(n_pre + m) * n, n, coeffs.p + (size_t)(n_pre + m) * n, n,
             cw.p + (size_t)(n_pre + m) * N, N, n_rel, small, big, offset_pows, st);
    build_qm31_trees(cw.p + (size_t)(n_pre + m) * N, N, tree_ptrs(trees, n_pre + m, n_pre + m + n_rel).data(), n_rel,
                     st);
    const std::vector<Digest> aroots = roots_of(trees, n_pre + m, n_pre + m + n_rel, st);
    for (uint32_t r = 0; r < n_rel; ++r) {
      acc_roots.push_back(aroots[r]);
      ch.absorb(acc_roots.back());
    }
  }
  proof.digests(trace_roots);
  if (n_pre > 0) {
    proof.u8(1);
    proof.digests(pre_roots);
  } else {
    proof.u8(0);
  }
  if (n_rel > 0) {
    proof.u8(1);
    proof.digests(acc_roots);
  } else {
    proof.u8(0);
  }

  // ---- constraint weights and the quotient -------------------------------------
  std::vector<qm31> alphas(n_trans_total);
  for (auto& a : alphas) a = ch.sample_q();
  std::vector<Boundary> bnd;
  air.boundary(n, bnd);
  for (uint32_t r = 0; r < n_rel; ++r) bnd.push_back({m + r, 0, qzero()});
  std::vector<qm31> betas(total_bound);
  for (auto& b : betas) b = ch.sample_q();
  if (wide) {
    ml_set_weights(*ml, air, alphas, betas);
  } else {
    for (uint32_t t = 0; t < n_trans_total; ++t) kc.alphas[t] = alphas[t];
    for (uint32_t b = 0; b < total_bound; ++b) {
      kc.betas[b] = betas[b];
      kc.b_col[b] = bnd[b].column;
      kc.b_val[b] = bnd[b].value;
      kc.b_pt[b] = qpow(w, bnd[b].step);
    }
    group_boundaries(kc);
  }
  // Z_H(d_i) = offset^n * (w_N^n)^(i mod 2^lb) - 1, and the stacked Rescue AIR's
  // y_i = d_i^(n/8) = offset^(n/8) (w_N^(n/8))^i, which repeats with period 8 * 2^lb
  const uint32_t period = air.id == AIR_RESCUE_STACKED ? 8u << lb : 0;
  kc.per_mask = period ? period - 1 : 0;
  kc.on = qpow(offset, n);
  if (!wide)
    if (const char* bad = quot_consts_out_of_range(kc, shift)) throw Error(ZS_EGENERIC, bad);
  h2d_small(d_kc.p, &kc, sizeof(kc), st);
  DevBuf<qm31> zh_tab((size_t)2 * shift, st), per_tab(period ? (size_t)5 * period : 1, st);
  {
    const uint32_t cnt = std::max<uint32_t>(shift, period);
    k_quot_tables<<<(cnt + kT - 1) / kT, kT, 0, st>>>(zh_tab.p, period ? per_tab.p : nullptr, d_kc.p,
                                                      q_root_of_unity(lb), q_root_of_unity(lN), period);
  }
  DevBuf<qm31> q(N, st);
  if (wide) {
    h2d_small(d_ml->p, ml.get(), sizeof(MlConsts), st);
    k_ml_quotient<<<(N + kT - 1) / kT, kT, 0, st>>>(cw.p, q.p, big.fwd, d_ml->p, zh_tab.p);
  } else if (RescueQuot rq; rescue_quot(kc, rq)) {
    k_quotient_rescue<<<(N + kT - 1) / kT, kT, 0, st>>>(cw.p, q.p, big.fwd, d_kc.p, rq, zh_tab.p, per_tab.p);
  } else {
    k_quotient<<<(N + kT - 1) / kT, kT, 0, st>>>(cw.p, q.p, big.fwd, d_kc.p, zh_tab.p, per_tab.p);
  }
  ZS_CUDA(cudaGetLastError());
  OwnedTree qtree(lN, st);
  build_qm31_tree(q.p, qtree.t, st);
  const Digest qroot = root_of(qtree.t, st);
  ch.absorb(qroot);
  proof.digest(qroot);

  // ---- DEEP evaluations (stark.zig:547-570) ------------------------------------
  const qm31 z = ch.sample_q();
  const qm31 wz = qmul(z, w);
  std::vector<qm31> deep(n_deep);
  std::vector<qm31> pre_z(n_pre);
  {
    DevBuf<qm31> zpow((size_t)2 * n, st);
    qm31_powers(z, zpow.p, n, st);
    qm31_powers(wz, zpow.p + n, n, st);
    const uint32_t nblk = (n + kT * kEvalPer - 1) / (kT * kEvalPer);
    DevBuf<qm31> partial((size_t)2 * ncol * nblk, st), sums((size_t)2 * ncol, st);
    k_eval_partial<<<dim3(nblk, ncol, 2), kT, 0, st>>>(coeffs.p, n, tl, zpow.p, 2, partial.p);
    k_eval_sum<<<2 * ncol, kT, 0, st>>>(partial.p, nblk, sums.p);
    ZS_CUDA(cudaGetLastError());
    std::vector<qm31> hs(2 * ncol);
    d2h_small(hs.data(), sums.p, hs.size() * sizeof(qm31), st);
    for (uint32_t j = 0; j < m_total; ++j) {
      deep[j] = hs[n_pre + j];                  // f_j(z)
      deep[m_total + j] = hs[ncol + n_pre + j];  // f_j(w z)
    }
    for (uint32_t j = 0; j < n_pre; ++j) pre_z[j] = hs[j];
    // computeQuotientAt (stark.zig:794-849)
    const qm31 zh = qsub(qpow(z, n), qone());
    const qm31 h = wide ? ml_composition(*ml, z, deep.data(), deep.data() + m_total, pre_z.data(), zh, false)
                        : composition(kc, z, deep.data(), deep.data() + m_total, pre_z.data(), zh);
    deep[2 * m_total] = qmul(h, qinv(zh));
  }
  for (auto& v : deep) ch.absorb(v);
  proof.qs(deep);

  // ---- DEEP codeword and FRI ---------------------------------------------------
  DeepConsts dc{};
  dc.m_total = m_total, dc.n_pre = n_pre, dc.shift = shift, dc.log_N = lN;
  dc.offset = offset, dc.z = z, dc.qz = deep[2 * m_total];
  std::vector<qm31> ge(n_deep + 2 * m_total);  // gammas, then f_j(z), f_j(wz)
  for (uint32_t j = 0; j < n_deep; ++j) ge[j] = ch.sample_q();
  for (uint32_t j = 0; j < 2 * m_total; ++j) ge[n_deep + j] = deep[j];
  DevBuf<DeepConsts> d_dc(1, st);
  h2d_small(d_dc.p, &dc, sizeof(dc), st);
  DevBuf<qm31> d_ge(ge.size(), st);
  h2d_small(d_ge.p, ge.data(), ge.size() * sizeof(qm31), st);
  std::vector<std::unique_ptr<DevBuf<qm31>>> layers;
  layers.push_back(std::make_unique<DevBuf<qm31>>(N, st));
  k_deep<<<(N + kT - 1) / kT, kT, 0, st>>>(cw.p, q.p, big.fwd, d_dc.p, d_ge.p, layers[0]->p);
  ZS_CUDA(cudaGetLastError());

  std::unique_ptr<FoldTables> ftabs_own;
  const FoldTables& ftabs = fold_tables(lN, st, ftabs_own);
  std::vector<std::unique_ptr<OwnedTree>> ftrees;
  for (unsigned i = 0; i < L; ++i) ftrees.push_back(std::make_unique<OwnedTree>(lN - i, st));
  // The commit phase (fri.zig:195-227) runs without host round trips: per layer a
  // one-thread kernel absorbs the layer's root into the device copy of the transcript
  // and samples the folding challenge, which the fold reads from device memory. The
  // layers of at most kTailMax values are committed and folded by one CTA (fri_tail).
  unsigned tail = L;  // first layer of the tail
  for (unsigned i = 0; i < L; ++i)
    if ((N >> i) <= kTailMax) {
      tail = i;
      break;
    }
  if (L - tail > kTailLayers) tail = L - kTailLayers;
  if (tail > 0) build_qm31_tree(layers[0]->p, ftrees[0]->t, st);
  std::vector<Digest> froots(L);
  // remainder (fri.zig:228-233): interpolate the first 2^(remainder_log - log_blowup)
  // points of layer L on the host (at most a few dozen values); they come back with
  // the transcript state and the layer roots, in one wait.
  const uint32_t rem = 1u << (fp.remainder_log - fp.log_blowup);
  std::vector<qm31> last(rem);
  if (L > 0) {
    DevBuf<Channel> d_ch(1, st);
    h2d_small(d_ch.p, &ch, sizeof(Channel), st);
    DevBuf<qm31> d_alpha(L, st);
    DevBuf<uint32_t> d_roots((size_t)8 * L, st);
    for (unsigned i = 0; i < tail; ++i) {
      k_fri_transcript<<<1, 32, 0, st>>>(d_ch.p, ftrees[i]->t.root(), d_roots.p + 8 * i, d_alpha.p + i);
      ZS_CUDA(cudaGetLastError());
      const uint32_t half = N >> (i + 1);
      layers.push_back(std::make_unique<DevBuf<qm31>>(half, st));
      fri_fold(layers[i]->p, layers[i + 1]->p, half, d_alpha.p + i, i, ftabs,
               i + 1 < tail ? &ftrees[i + 1]->t : nullptr, st);
    }
    DevBuf<FriTail> d_tail(1, st);
    if (tail < L) {
      FriTail ft{};
      ft.first = tail, ft.count = L - tail, ft.log_size = lN - tail, ft.tables = ftabs.tables;
      for (unsigned i = tail; i < L; ++i) layers.push_back(std::make_unique<DevBuf<qm31>>(N >> (i + 1), st));
      for (unsigned c = 0; c <= ft.count; ++c) ft.layer[c] = layers[tail + c]->p;
      for (unsigned c = 0; c < ft.count; ++c) {
        ft.off_inv[c] = ftabs.offset_inv(tail + c);
        ft.tree[c] = ftrees[tail + c]->t.words;
      }
      ft.roots = d_roots.p + 8 * tail;
      ft.alphas = d_alpha.p + tail;
      h2d_small(d_tail.p, &ft, sizeof(ft), st);
      fri_tail(d_tail.p, d_ch.p, st);
    }
    std::vector<uint32_t> words((size_t)8 * L);
    const D2H back[3] = {{&ch, d_ch.p, sizeof(Channel)},  // the transcript continues on the host
                         {words.data(), d_roots.p, words.size() * sizeof(uint32_t)},
                         {last.data(), layers[L]->p, rem * sizeof(qm31)}};
    d2h_many(back, 3, st);
    for (unsigned i = 0; i < L; ++i)
      for (int b = 0; b < 32; ++b) froots[i][b] = (uint8_t)(words[8 * i + b / 4] >> (8 * (b % 4)));
  } else {
    d2h_small(last.data(), layers[L]->p, rem * sizeof(qm31), st);
  }
  std::vector<qm31> xs(rem);
  {
    const qm31 wl = q_root_of_unity(lN - L);
    qm31 acc = qpow(offset, (uint64_t)1 << L);
    for (uint32_t j = 0; j < rem; ++j) {
      xs[j] = acc;
      acc = qmul(acc, wl);
    }
  }
  const std::vector<qm31> remainder = interpolate_small(xs, last);
  for (auto& v : remainder) ch.absorb(v);

  // ---- queries (fri.zig:236-256, stark.zig:595-625) -----------------------------
  // Every revealed value and Merkle sibling is gathered by one kernel, in the order the
  // proof lists them, so serialization copies contiguous runs of the gathered words. The
  // gather list is the same for every query but for the positions, so the host builds
  // one query's template and the kernel applies it to all of them.
  std::vector<uint64_t> p0s(sp.num_queries);
  for (auto& p : p0s) p = ch.sample_index(N);
  std::vector<QueryReq> tmpl;
  uint32_t sec_words[2] = {0, 0};
  auto want = [&](int sec, const void* base, uint32_t words, uint8_t mode, unsigned modlog, uint8_t lvl) {
    tmpl.push_back({reinterpret_cast<const uint32_t*>(base), sec_words[sec], (uint16_t)words, (uint8_t)sec, mode,
                    (uint8_t)modlog, lvl});
    sec_words[sec] += words;
  };
  auto want_path = [&](int sec, const DeviceTree& t, uint8_t mode, unsigned modlog) {
    for (unsigned lvl = 0; lvl < t.log_n; ++lvl) want(sec, t.level(lvl), 8, mode, modlog, (uint8_t)lvl);
  };
  // FRI pairs, per query: per layer i the two values at p0 mod 2^(lN-i-1) and that plus
  // 2^(lN-i-1), then their two paths
  for (unsigned i = 0; i < L; ++i) {
    const unsigned ml = lN - (i + 1);
    want(0, layers[i]->p, 4, kQLow, ml, kQValue);
    want(0, layers[i]->p, 4, kQHigh, ml, kQValue);
    want_path(0, ftrees[i]->t, kQLow, ml);
    want_path(0, ftrees[i]->t, kQHigh, ml);
  }
  // STARK reveals, per query: the values (columns at p0, columns at p0 + shift, the
  // quotient, preprocessed columns), then their paths in the same order
  for (uint32_t j = 0; j < m_total; ++j) want(1, cw.p + (size_t)(n_pre + j) * N, 4, kQP0, lN, kQValue);
  for (uint32_t j = 0; j < m_total; ++j) want(1, cw.p + (size_t)(n_pre + j) * N, 4, kQShift, lN, kQValue);
  want(1, q.p, 4, kQP0, lN, kQValue);
  for (uint32_t j = 0; j < n_pre; ++j) want(1, cw.p + (size_t)j * N, 4, kQP0, lN, kQValue);
  for (uint32_t j = 0; j < m_total; ++j) want_path(1, trees[n_pre + j]->t, kQP0, lN);
  for (uint32_t j = 0; j < m_total; ++j) want_path(1, trees[n_pre + j]->t, kQShift, lN);
  want_path(1, qtree.t, kQP0, lN);
  for (uint32_t j = 0; j < n_pre; ++j) want_path(1, trees[j]->t, kQP0, lN);
  const uint32_t nq = (uint32_t)sp.num_queries;
  const size_t off = (size_t)nq * (sec_words[0] + sec_words[1]);
  std::vector<uint32_t> gathered(off);
  if (off > 0) {
    DevBuf<QueryReq> d_tmpl(tmpl.size(), st);
    DevBuf<uint64_t> d_p0s(nq, st);
    DevBuf<uint32_t> d_out(off, st);
    h2d_small(d_tmpl.p, tmpl.data(), tmpl.size() * sizeof(QueryReq), st);
    h2d_small(d_p0s.p, p0s.data(), nq * sizeof(uint64_t), st);
    for (uint32_t q0 = 0; q0 < nq; q0 += 65535) {  // grid.y is at most 65535
      const dim3 grid(((uint32_t)tmpl.size() + kT - 1) / kT, std::min<uint32_t>(65535, nq - q0));
      k_gather_queries<<<grid, kT, 0, st>>>(d_tmpl.p, (uint32_t)tmpl.size(), d_p0s.p, q0, nq, shift, lN,
                                            sec_words[0], sec_words[1], d_out.p);
    }
    ZS_CUDA(cudaGetLastError());
    d2h_small(gathered.data(), d_out.p, off * sizeof(uint32_t), st);
  }
  size_t cursor = 0;
  auto put_values = [&](size_t count) {  // QM31 values: 4 words each, as on the wire
    proof.bytes(gathered.data() + cursor, 16 * count);
    cursor += 4 * count;
  };
  auto put_path = [&](unsigned log_n) {  // []Digest: u64 length, 32 bytes per digest
    proof.u64(log_n);
    proof.bytes(gathered.data() + cursor, (size_t)32 * log_n);
    cursor += (size_t)8 * log_n;
  };

  // ---- serialization (stark.zig:107-122, fri.zig:72-79) --------------------------
  proof.out.reserve(proof.out.size() + (size_t)off * 4 + (size_t)sp.num_queries * (L + reveal_len) * 16 +
                    (size_t)32 * (L + 64) + 1024);
  proof.u8(fp.log_size);  // Fri.Proof.params
  proof.u8(fp.log_blowup);
  proof.u64(fp.num_queries);
  proof.u8(fp.remainder_log);
  proof.digests(froots);
  proof.qs(remainder);
  proof.u64(sp.num_queries);
  for (uint64_t qi = 0; qi < sp.num_queries; ++qi) {
    proof.u64(p0s[qi]);
    proof.u64(L);
    for (unsigned i = 0; i < L; ++i) {
      put_values(2);
      put_path(lN - i);
      put_path(lN - i);
    }
  }
  proof.u64(sp.num_queries);
  for (uint64_t qi = 0; qi < sp.num_queries; ++qi) {
    proof.u64(p0s[qi]);
    proof.u64(reveal_len);
    put_values(reveal_len);
    proof.u64(reveal_len);
    for (uint32_t k = 0; k < reveal_len; ++k) put_path(lN);
  }
  ZS_CUDA(cudaStreamSynchronize(st));
  return proof.out;
}

// The commitment of columns alone (stark.zig:397-414): interpolate each column on
// H, evaluate on D, one Merkle tree of hashQM31 leaves per column; returns the roots
// as a wire []Digest (u64 count, then 32 bytes per column).
std::vector<uint8_t> commit_columns(const uint8_t* cols_b, size_t cols_len, unsigned trace_log, unsigned log_blowup,
                                    cudaStream_t st) {
  const WireColumns cols = locate_columns(cols_b, cols_len);
  const unsigned lN = trace_log + log_blowup;
  if (lN > 26) throw Error(ZS_EMALFORMED, "trace_log + log_blowup above 26");
  const uint32_t n = 1u << trace_log, N = 1u << lN, C = (uint32_t)cols.size();
  for (uint64_t l : cols.len)
    if (l != n) throw Error(ZS_EMALFORMED, "column length is not 2^trace_log");
  retain_pool_memory();
  PinnedScope pinned(st);
  WireWriter out;
  out.u64(C);
  if (C == 0) return out.out;
  std::unique_ptr<NttTables> small_own, big_own;
  std::unique_ptr<DevBuf<qm31>> pows_own;
  const NttTables& small = ntt_tables(trace_log, st, small_own);
  const NttTables& big = ntt_tables(lN, st, big_own);
  const qm31* offset_pows = offset_powers(trace_log, st, pows_own);
  DevBuf<qm31> vals((size_t)C * n, st), coeffs((size_t)C * n, st), cw((size_t)C * N, st);
  upload_columns(cols, vals.p, n, st);
  lde_qm31(vals.p, n, coeffs.p, n, cw.p, N, C, small, big, offset_pows, st);
  // trees of up to 1 GiB in all are built together, then their roots read back
  const size_t tree_bytes = DeviceTree::words_for(lN) * sizeof(uint32_t);
  const uint32_t per = (uint32_t)std::max<size_t>(1, std::min<size_t>(kTreeBatch, ((size_t)1 << 30) / tree_bytes));
  std::vector<std::unique_ptr<OwnedTree>> trees;
  for (uint32_t j = 0; j < std::min(per, C); ++j) trees.push_back(std::make_unique<OwnedTree>(lN, st));
  for (uint32_t c0 = 0; c0 < C; c0 += per) {
    const uint32_t c = std::min(per, C - c0);
    build_qm31_trees(cw.p + (size_t)c0 * N, N, tree_ptrs(trees, 0, c).data(), c, st);
    for (const Digest& d : roots_of(trees, 0, c, st)) out.digest(d);
  }
  return out.out;
}

}  // namespace zs
