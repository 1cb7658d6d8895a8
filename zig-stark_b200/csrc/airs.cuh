// AIRs compiled into the backend, in the shape GenericStark expects
// (src/m31/stark.zig:45-74): counts, evalTransition(x, current, next, out),
// boundaryAssertions(public, n, out), maxConstraintDegree(n) and optional LogUp
// metadata. A comptime Zig AIR cannot cross a C ABI, so the AIR is selected by id
// (include/zs_m31.h) and its PublicInputs arrive in wire form.
//
// evalTransition is __host__ __device__: the quotient kernel evaluates it on D, the
// host evaluates it once at z for computeQuotientAt (stark.zig:794-849).
#pragma once
#include <cstring>
#include <vector>

#include "common.cuh"

namespace zs {

enum AirIdInternal : uint32_t {
  AIR_FIB = 0,
  AIR_SEEDED_FIB = 1,
  AIR_RANGE_CHECK = 2,
  AIR_AND_TABLE = 3,
  AIR_MULTIPLICITY = 4,
  AIR_RESCUE_EXAMPLE = 5,
  AIR_LINEAR_EXAMPLE = 6,
  AIR_RESCUE_STACKED = 7,
  AIR_ML_LINEAR = 8,
  AIR_COUNT = 9,
};

// Limits of the generic quotient path, which keeps a row's columns in per-thread
// arrays. The linear-layer AIR (AIR_ML_LINEAR) is wider and has kernels of its own
// that stream its columns (constraints.cuh, stark.cu).
constexpr unsigned kMaxCols = 16;      // main + accumulator columns
constexpr unsigned kMaxTrans = 16;     // AIR transition constraints
constexpr unsigned kMaxBound = 16;     // boundary assertions incl. synthesized ones
constexpr unsigned kMaxPre = 4;
constexpr unsigned kMaxRel = 2;
constexpr unsigned kMaxKey = 4;

// The linear-layer AIR: y = W x with W 128 x 128 (public input), input vectors bound
// by one LogUp relation to a preprocessed input table. Columns x_0..x_127, y_0..y_127,
// sel, mult; preprocessed P_0..P_127.
constexpr uint32_t kMlDim = 128;
constexpr uint32_t kMlSel = 2 * kMlDim, kMlMult = 2 * kMlDim + 1, kMlCols = 2 * kMlDim + 2;

// Constants an AIR's evalTransition needs (row-dependent polynomials of the examples).
struct AirConsts {
  uint32_t id;
  uint32_t poly_len;
  qm31 poly[4][8];  // rescue: rc_poly[j] (main.zig:87-111); linear: inc (main.zig:59-81);
                    // stacked rescue: P_j, the periodic round constants on <w8>
  qm31 w8_7;        // stacked rescue: w8^7, the row phase whose round is switched off
  uint64_t n_div8;  // stacked rescue: n / 8
};

// Rescue example MDS matrix (examples/rescue/src/main.zig:19-25): circulant with first
// row (2, 3, 1, 1), so entry (j, l) is first[(l - j) mod 4].
ZS_HD uint32_t rescue_mds(int j, int l) {
  const uint32_t first = 0x01010302u;  // bytes 2, 3, 1, 1
  return (first >> (8 * ((l - j) & 3))) & 0xff;
}

ZS_HD qm31 horner(const qm31* c, uint32_t len, const qm31& x) {
  qm31 r = qzero();
  for (uint32_t i = len; i > 0; --i) r = qadd(qmul(r, x), c[i - 1]);
  return r;
}
ZS_HD qm31 qpow5(const qm31& v) {
  const qm31 v2 = qmul(v, v);
  return qmul(qmul(v2, v2), v);
}

// The transition constraints of each AIR.
ZS_HD void air_eval(const AirConsts& k, const qm31& x, const qm31* cur, const qm31* next, qm31* out) {
  switch (k.id) {
    case AIR_FIB:
    case AIR_SEEDED_FIB:  // stark.zig:886-892
      out[0] = qsub(next[0], cur[1]);
      out[1] = qsub(qsub(next[1], cur[0]), cur[1]);
      break;
    case AIR_RESCUE_EXAMPLE:  // examples/rescue/src/main.zig:113-123
      for (int j = 0; j < 4; ++j) {
        qm31 expect = qzero();
        for (int l = 0; l < 4; ++l) expect = qadd(expect, qmul_m(qpow5(cur[l]), rescue_mds(j, l)));
        expect = qadd(expect, horner(k.poly[j], k.poly_len, x));
        out[j] = qsub(next[j], expect);
      }
      break;
    case AIR_RESCUE_STACKED: {
      // Permutations of 8 rows; s_j = cur[j], q_j = cur[4 + j] = s_j^2 and
      // t_j = cur[8 + j] = q_j s_j, so the round s^5 = t q has degree 2.
      // y = x^(n/8) is w8^(r mod 8) on row r; the factor y - w8^7 switches the round
      // off on each permutation's last row, and the round constants are P_j(y).
      const qm31 y = qpow(x, k.n_div8);
      const qm31 z = qsub(y, k.w8_7);
      for (int j = 0; j < 4; ++j) {
        qm31 expect = qzero();
        for (int l = 0; l < 4; ++l) expect = qadd(expect, qmul_m(qmul(cur[8 + l], cur[4 + l]), rescue_mds(j, l)));
        expect = qadd(expect, horner(k.poly[j], 8, y));
        out[j] = qmul(z, qsub(next[j], expect));
        out[4 + j] = qsub(cur[4 + j], qmul(cur[j], cur[j]));
        out[8 + j] = qsub(cur[8 + j], qmul(cur[4 + j], cur[j]));
      }
      break;
    }
    case AIR_LINEAR_EXAMPLE:  // examples/ml_linear/src/main.zig:84-87
      out[0] = qsub(qsub(next[0], cur[0]), horner(k.poly[0], k.poly_len, x));
      break;
    default:  // lookup AIRs have no transition constraints
      break;
  }
}

// The stacked Rescue transitions with the row-periodic values read from `per`
// ({y - w8^7, P_0(y), ..., P_3(y)} for y = x^(n/8)), which the quotient kernel takes from
// a table instead of raising every domain point to n/8. Same values as air_eval.
ZS_HD void rescue_stacked_eval(const qm31* per, const qm31* cur, const qm31* next, qm31* out) {
  const qm31 z = per[0];
  qm31 s5[4];  // t_l q_l = s_l^5, once per column
#pragma unroll
  for (int l = 0; l < 4; ++l) s5[l] = qmul(cur[8 + l], cur[4 + l]);
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    qm31 expect = per[1 + j];
#pragma unroll
    for (int l = 0; l < 4; ++l) expect = qadd(expect, qmul_m(s5[l], rescue_mds(j, l)));
    out[j] = qmul(z, qsub(next[j], expect));
    out[4 + j] = qsub(cur[4 + j], qmul(cur[j], cur[j]));
    out[8 + j] = qsub(cur[8 + j], qmul(cur[4 + j], cur[j]));
  }
}

struct Boundary {
  uint32_t column;
  uint64_t step;
  qm31 value;
};

// Host-side description of an AIR instance (counts, LogUp metadata, boundaries).
struct AirInfo {
  uint32_t id = 0;
  uint32_t m = 0, num_trans = 0, num_bound = 0, n_pre = 0, n_lc = 0, n_rel = 0;
  uint32_t fixed_n = 0;  // 0 = any trace length
  uint32_t sel[kMaxRel] = {}, mult[kMaxRel] = {};
  uint32_t n_keys[kMaxRel] = {}, keys[kMaxRel][kMaxKey] = {}, tabs[kMaxRel][kMaxKey] = {};
  uint64_t dc_mul = 1;  // maxConstraintDegree(n) = dc_mul * (n - 1) (+ n/8 if dc_plus_n8)
  bool dc_plus_n8 = false;
  std::vector<qm31> pi;  // public inputs (QM31 fields in declaration order)
  std::vector<qm31> x_inputs;  // linear example: public x
  std::vector<uint32_t> w;     // linear layer: W, row-major kMlDim x kMlDim M31 values
  AirConsts consts{};

  uint64_t max_constraint_degree(uint64_t n) const {  // stark.zig:217-221 incl. LogUp padding
    uint64_t d = dc_mul * (n - 1) + (dc_plus_n8 ? n / 8 : 0);
    if (n_rel > 0 && 3 * (n - 1) > d) d = 3 * (n - 1);
    return d;
  }
  void boundary(uint64_t n, std::vector<Boundary>& out) const;
};

// Parses `air_id` and its PublicInputs (wire form); throws Error(-2) on malformed input.
AirInfo make_air(uint32_t air_id, const uint8_t* pi, size_t pi_len);

}  // namespace zs
