// ORACLE — test infrastructure only. AIRs in the shape GenericStark expects
// (src/m31/stark.zig:45-74): column/constraint/boundary counts,
// evalTransition(x, current, next, out), boundaryAssertions(public, n, out),
// maxConstraintDegree(n) and the optional LogUp metadata.
//
// Reference AIRs restated here:
//   FibAir            src/m31/stark.zig:877-931
//   RangeCheckAir     src/m31/stark.zig:964-1041
//   AndTableAir       src/m31/stark.zig:1048-1131
//   MultiplicityAir   src/m31/stark.zig:1139-1216
//   RescueAir (n=8)   examples/rescue/src/main.zig:13-144
//   LinearAir (n=8)   examples/ml_linear/src/main.zig:21-116
// AIRs for workloads the reference has no AIR for, written in the same shape:
//   SeededFibAir      FibAir with public a_0, a_1 (boundaries from public inputs)
//   RescueStackedAir  independent Rescue permutations stacked 8 rows each
//   MlLinearAir       y = W x for a batch of input vectors bound by LogUp to a
//                     preprocessed input table (examples/ml_linear widened)
#pragma once
#include <memory>
#include <stdexcept>
#include <vector>

#include "poly.hpp"
#include "wire.hpp"

namespace orc {

// stark.zig:12-17.
struct BoundaryAssertion {
  size_t column;
  size_t step;
  QM31 value;
};

enum AirId : uint32_t {
  AIR_FIB = 0,
  AIR_SEEDED_FIB = 1,
  AIR_RANGE_CHECK = 2,
  AIR_AND_TABLE = 3,
  AIR_MULTIPLICITY = 4,
  AIR_RESCUE_EXAMPLE = 5,
  AIR_LINEAR_EXAMPLE = 6,
  AIR_RESCUE_STACKED = 7,
  AIR_ML_LINEAR = 8,
};

struct Air {
  virtual ~Air() = default;
  size_t num_columns = 0, num_transitions = 0, num_boundary = 0;
  size_t num_preprocessed = 0, num_lookup_columns = 0, num_lookup_relations = 0;
  std::vector<size_t> selector_cols, mult_cols;
  std::vector<std::vector<size_t>> key_cols, table_cols;
  virtual void evalTransition(const QM31& x, const QM31* cur, const QM31* next, QM31* out) const = 0;
  virtual size_t maxConstraintDegree(size_t n) const = 0;
  virtual void boundaryAssertions(size_t n, BoundaryAssertion* out) const = 0;
  // Rejects a trace length the AIR cannot be used with.
  virtual void checkTraceLen(size_t) const {}
};

// stark.zig:877-904.
struct FibAir : Air {
  QM31 claimed;
  explicit FibAir(QM31 c) : claimed(c) {
    num_columns = 2;
    num_transitions = 2;
    num_boundary = 3;
  }
  void evalTransition(const QM31&, const QM31* cur, const QM31* next, QM31* out) const override {
    out[0] = next[0].sub(cur[1]);
    out[1] = next[1].sub(cur[0]).sub(cur[1]);
  }
  size_t maxConstraintDegree(size_t n) const override { return n - 1; }
  void boundaryAssertions(size_t n, BoundaryAssertion* out) const override {
    out[0] = {0, 0, QM31::zero()};
    out[1] = {1, 0, QM31::one()};
    out[2] = {0, n - 1, claimed};
  }
};

// FibAir with a_0 and a_1 taken from the public inputs (a_0 = 1 and a seeded
// a_1 for the 2^12-row Fibonacci workload). Public inputs: {a0, a1, claimed}.
struct SeededFibAir : FibAir {
  QM31 a0, a1;
  SeededFibAir(QM31 x0, QM31 x1, QM31 c) : FibAir(c), a0(x0), a1(x1) {}
  void boundaryAssertions(size_t n, BoundaryAssertion* out) const override {
    out[0] = {0, 0, a0};
    out[1] = {1, 0, a1};
    out[2] = {0, n - 1, claimed};
  }
};

// stark.zig:964-1216 (three lookup AIRs with no transitions or boundaries).
struct LookupAir : Air {
  LookupAir(size_t n_pre, size_t n_lc, std::vector<size_t> keys, std::vector<size_t> tabs,
            size_t sel, size_t mult) {
    num_columns = 3;
    num_preprocessed = n_pre;
    num_lookup_columns = n_lc;
    num_lookup_relations = 1;
    selector_cols = {sel};
    key_cols = {keys};
    table_cols = {tabs};
    mult_cols = {mult};
  }
  void evalTransition(const QM31&, const QM31*, const QM31*, QM31*) const override {}
  size_t maxConstraintDegree(size_t n) const override { return n - 1; }
  void boundaryAssertions(size_t, BoundaryAssertion*) const override {}
};

// examples/rescue/src/main.zig: s = 4, n = 8, MDS circulant (2,3,1,1), x^5
// sbox, LCG round constants, round-constant polynomials interpolated on H.
struct RescueExampleAir : Air {
  static constexpr size_t S = 4, N = 8, ROUNDS = N - 1;
  static constexpr uint32_t MDS[4][4] = {{2, 3, 1, 1}, {1, 2, 3, 1}, {1, 1, 2, 3}, {3, 1, 1, 2}};
  QM31 initial[4], final_[4];
  std::vector<QM31> rc_poly[4];

  static void roundConstants(QM31 rc[ROUNDS][S]) {  // main.zig:28-38
    uint64_t seed = 0x243f6a8885a308d3ull;
    for (size_t r = 0; r < ROUNDS; ++r)
      for (size_t j = 0; j < S; ++j) {
        seed = seed * 6364136223846793005ull + 1442695040888963407ull;
        rc[r][j] = QM31::fromM31(M31::fromInt((uint32_t)(seed >> 33)));
      }
  }
  static void applyRound(size_t r, const QM31 st[S], QM31 out[S]) {  // main.zig:41-52
    QM31 rc[ROUNDS][S];
    roundConstants(rc);
    QM31 boxed[S];
    for (size_t j = 0; j < S; ++j) boxed[j] = st[j].pow(5);
    for (size_t j = 0; j < S; ++j) {
      QM31 acc = QM31::zero();
      for (size_t l = 0; l < S; ++l) acc = acc.add(boxed[l].mul(QM31::fromU32(MDS[j][l])));
      out[j] = acc.add(rc[r][j]);
    }
  }
  RescueExampleAir(const QM31* init, const QM31* fin) {
    num_columns = S;
    num_transitions = S;
    num_boundary = 2 * S;
    for (size_t j = 0; j < S; ++j) {
      initial[j] = init[j];
      final_[j] = fin[j];
    }
    // main.zig:87-111 prepare(): interpolate rc columns on H (n = 8).
    QM31 rc[ROUNDS][S];
    roundConstants(rc);
    QM31 w = QM31::primitiveRootOfUnity(3);
    std::vector<QM31> h(N);
    QM31 acc = QM31::one();
    for (size_t r = 0; r < N; ++r) {
      h[r] = acc;
      acc = acc.mul(w);
    }
    for (size_t j = 0; j < S; ++j) {
      std::vector<QM31> ys(N);
      for (size_t r = 0; r < N; ++r) ys[r] = r < ROUNDS ? rc[r][j] : QM31::zero();
      rc_poly[j] = interpolateLagrange(h, ys);
    }
  }
  void evalTransition(const QM31& x, const QM31* cur, const QM31* next, QM31* out) const override {
    for (size_t j = 0; j < S; ++j) {  // main.zig:113-123
      QM31 expect = QM31::zero();
      for (size_t l = 0; l < S; ++l)
        expect = expect.add(cur[l].pow(5).mul(QM31::fromU32(MDS[j][l])));
      expect = expect.add(evalHorner(rc_poly[j], x));
      out[j] = next[j].sub(expect);
    }
  }
  size_t maxConstraintDegree(size_t n) const override { return 5 * (n - 1); }
  void boundaryAssertions(size_t n, BoundaryAssertion* out) const override {
    for (size_t j = 0; j < S; ++j) {
      out[j] = {j, 0, initial[j]};
      out[S + j] = {j, n - 1, final_[j]};
    }
  }
  void checkTraceLen(size_t n) const override {
    if (n != N) throw WireError("rescue example AIR is defined for 8 rows", -1);
  }
};

// examples/ml_linear/src/main.zig: a dot product of 8 fixed weights with the
// public input x, as a running-sum column; increments interpolated on H.
struct LinearExampleAir : Air {
  static constexpr size_t N = 8;
  std::vector<QM31> x;
  QM31 claimed_y;
  std::vector<QM31> inc;
  static QM31 weight(size_t r) { return QM31::fromU32((uint32_t)(r + 1)); }
  LinearExampleAir(std::vector<QM31> xs, QM31 y) : x(std::move(xs)), claimed_y(y) {
    num_columns = 1;
    num_transitions = 1;
    num_boundary = 2;
    if (x.size() != N) throw WireError("linear example AIR takes 8 inputs", -2);
    QM31 w = QM31::primitiveRootOfUnity(3);  // main.zig:59-81
    std::vector<QM31> h(N), ys(N);
    QM31 acc = QM31::one();
    for (size_t r = 0; r < N; ++r) {
      h[r] = acc;
      acc = acc.mul(w);
    }
    for (size_t r = 0; r < N; ++r) ys[r] = weight((r + 1) % N).mul(x[(r + 1) % N]);
    inc = interpolateLagrange(h, ys);
  }
  void evalTransition(const QM31& xp, const QM31* cur, const QM31* next, QM31* out) const override {
    out[0] = next[0].sub(cur[0]).sub(evalHorner(inc, xp));  // main.zig:84-87
  }
  size_t maxConstraintDegree(size_t n) const override { return n - 1; }
  void boundaryAssertions(size_t n, BoundaryAssertion* out) const override {
    out[0] = {0, 0, weight(0).mul(x[0])};
    out[1] = {0, n - 1, claimed_y};
  }
  void checkTraceLen(size_t n) const override {
    if (n != N) throw WireError("linear example AIR is defined for 8 rows", -1);
  }
};

// Independent Rescue permutations (the example's round: x^5 sbox, circulant MDS
// (2,3,1,1), the example's LCG round constants) stacked 8 rows per permutation.
// Columns s_0..s_3 (state), q_j = s_j^2 and t_j = q_j s_j, so s^5 = t q and every
// constraint has degree 2 in the columns:
//   C_j     = Z(x) * (next.s_j - sum_l MDS[j][l] * t_l * q_l - rc_j(x))   j < 4
//   C_{4+j} = q_j - s_j^2,   C_{8+j} = t_j - q_j s_j
// with y = x^(n/8) (so y = w8^(r mod 8) on row r), Z(x) = y - w8^7 switching the
// round off on the last row of every permutation, and rc_j(x) = P_j(y), P_j the
// degree-<8 interpolant of the round constants rc[t][j] (rc[7][j] = 0) on <w8>.
// maxConstraintDegree = 2(n-1) + n/8, so at blowup 4 the FRI code keeps rate 1/2.
// Boundaries: the first permutation's input and the last permutation's output.
// PublicInputs {initial: [4]QM31, final: [4]QM31}.
struct RescueStackedAir : Air {
  QM31 initial[4], final_[4];
  std::vector<QM31> P[4];  // P_j coefficients
  QM31 w8_7;
  mutable size_t trace_n = 8;
  RescueStackedAir(const QM31* init, const QM31* fin) {
    num_columns = 12;
    num_transitions = 12;
    num_boundary = 8;
    for (size_t j = 0; j < 4; ++j) {
      initial[j] = init[j];
      final_[j] = fin[j];
    }
    QM31 rc[7][4];
    RescueExampleAir::roundConstants(rc);
    QM31 w8 = QM31::primitiveRootOfUnity(3);
    std::vector<QM31> h(8);
    QM31 acc = QM31::one();
    for (size_t t = 0; t < 8; ++t) {
      h[t] = acc;
      acc = acc.mul(w8);
    }
    w8_7 = h[7];
    for (size_t j = 0; j < 4; ++j) {
      std::vector<QM31> ys(8);
      for (size_t t = 0; t < 8; ++t) ys[t] = t < 7 ? rc[t][j] : QM31::zero();
      P[j] = interpolateLagrange(h, ys);
    }
  }
  void evalTransition(const QM31& x, const QM31* cur, const QM31* next, QM31* out) const override {
    // y = x^(n/8); n is set by checkTraceLen before any evaluation
    QM31 y = x.pow(trace_n / 8);
    QM31 z = y.sub(w8_7);
    for (size_t j = 0; j < 4; ++j) {
      QM31 expect = QM31::zero();
      for (size_t l = 0; l < 4; ++l)
        expect = expect.add(cur[8 + l].mul(cur[4 + l]).mul(QM31::fromU32(RescueExampleAir::MDS[j][l])));
      expect = expect.add(evalHorner(P[j], y));
      out[j] = z.mul(next[j].sub(expect));
      out[4 + j] = cur[4 + j].sub(cur[j].mul(cur[j]));
      out[8 + j] = cur[8 + j].sub(cur[4 + j].mul(cur[j]));
    }
  }
  size_t maxConstraintDegree(size_t n) const override { return 2 * (n - 1) + n / 8; }
  void boundaryAssertions(size_t n, BoundaryAssertion* out) const override {
    for (size_t j = 0; j < 4; ++j) {
      out[j] = {j, 0, initial[j]};
      out[4 + j] = {j, n - 1, final_[j]};
    }
  }
  void checkTraceLen(size_t n) const override {
    if (n < 8) throw WireError("stacked rescue AIR needs at least 8 rows", -2);
    trace_n = n;
  }
};

// One linear layer y = W x over M31 (examples/ml_linear/src/main.zig:21-116 proves one
// dot product of public weights with public inputs; this is the same kind of statement
// for a 128 x 128 weight matrix and a batch of input vectors that stay private and
// are bound to a committed input table instead).
// Columns: x_0..x_127 (0..127), y_0..y_127 (128..255), sel (256), mult (257).
// Preprocessed: P_0..P_127, the input table (one input vector per table row).
// Rows with sel = 1 hold an input vector x and its output y = W x; rows with sel = 0
// are table rows (x = y = 0 there, P = a table vector).
//   C_k = y_k - sum_l W[k][l] x_l, k < 128 (every row; degree 1)
//   one LogUp relation: key (x_0..x_127) on rows with sel = 1, multiplicity `mult`,
//   against table key (P_0..P_127) on rows with sel = 0: every input vector is a row
//   of the committed input table (combined with 128 per-column challenges).
//   boundary: sel = 0 on the last row (the one row the transitions leave unchecked,
//   stark.zig:505-533 multiplies them by x - w^(n-1), must not carry an input).
// PublicInputs {w: []QM31, 128 x 128 row-major, each an M31 value}.
struct MlLinearAir : Air {
  static constexpr size_t D = 128;
  std::vector<M31> W;  // row-major D x D
  explicit MlLinearAir(const std::vector<QM31>& w) {
    if (w.size() != D * D) throw WireError("ml linear AIR takes a 128 x 128 weight matrix", -2);
    W.resize(D * D);
    for (size_t k = 0; k < D * D; ++k) {
      if (w[k].a.c1.v != 0 || w[k].b.c0.v != 0 || w[k].b.c1.v != 0)
        throw WireError("ml linear weights are M31 values", -2);
      W[k] = w[k].a.c0;
    }
    num_columns = 2 * D + 2;
    num_transitions = D;
    num_boundary = 1;
    num_preprocessed = D;
    num_lookup_columns = D;
    num_lookup_relations = 1;
    selector_cols = {2 * D};
    mult_cols = {2 * D + 1};
    std::vector<size_t> cols(D);
    for (size_t l = 0; l < D; ++l) cols[l] = l;
    key_cols = {cols};
    table_cols = {cols};
  }
  // v * w for an M31 weight w: each M31 component scaled (QM31.mul by fromM31(w)).
  static QM31 scale(const QM31& v, M31 w) {
    return QM31(CM31(v.a.c0.mul(w), v.a.c1.mul(w)), CM31(v.b.c0.mul(w), v.b.c1.mul(w)));
  }
  void evalTransition(const QM31&, const QM31* cur, const QM31*, QM31* out) const override {
    for (size_t k = 0; k < D; ++k) {
      QM31 acc = QM31::zero();
      for (size_t l = 0; l < D; ++l) acc = acc.add(scale(cur[l], W[k * D + l]));
      out[k] = cur[D + k].sub(acc);
    }
  }
  size_t maxConstraintDegree(size_t n) const override { return n - 1; }
  void boundaryAssertions(size_t n, BoundaryAssertion* out) const override { out[0] = {2 * D, n - 1, QM31::zero()}; }
  void checkTraceLen(size_t n) const override {
    if (n < 2) throw WireError("ml linear AIR needs at least 2 rows", -2);
  }
};

// Builds the AIR for `air_id` from the wire encoding of its PublicInputs.
inline std::unique_ptr<Air> makeAir(uint32_t air_id, const uint8_t* pi, size_t pi_len) {
  Reader r(pi, pi_len);
  std::unique_ptr<Air> air;
  switch (air_id) {
    case AIR_FIB: {
      QM31 c = r.qm31();
      air = std::make_unique<FibAir>(c);
      break;
    }
    case AIR_SEEDED_FIB: {
      QM31 a0 = r.qm31(), a1 = r.qm31(), c = r.qm31();
      air = std::make_unique<SeededFibAir>(a0, a1, c);
      break;
    }
    case AIR_RANGE_CHECK:
      air = std::make_unique<LookupAir>(1, 1, std::vector<size_t>{0}, std::vector<size_t>{0}, 2, 1);
      break;
    case AIR_AND_TABLE:
      air = std::make_unique<LookupAir>(2, 2, std::vector<size_t>{0, 1}, std::vector<size_t>{0, 1}, 2, 2);
      break;
    case AIR_MULTIPLICITY:
      air = std::make_unique<LookupAir>(1, 1, std::vector<size_t>{0}, std::vector<size_t>{0}, 2, 1);
      break;
    case AIR_RESCUE_EXAMPLE: {
      QM31 init[4], fin[4];
      for (auto& v : init) v = r.qm31();
      for (auto& v : fin) v = r.qm31();
      air = std::make_unique<RescueExampleAir>(init, fin);
      break;
    }
    case AIR_LINEAR_EXAMPLE: {
      std::vector<QM31> xs = r.qm31s();
      QM31 y = r.qm31();
      air = std::make_unique<LinearExampleAir>(std::move(xs), y);
      break;
    }
    case AIR_RESCUE_STACKED: {
      QM31 init[4], fin[4];
      for (auto& v : init) v = r.qm31();
      for (auto& v : fin) v = r.qm31();
      air = std::make_unique<RescueStackedAir>(init, fin);
      break;
    }
    case AIR_ML_LINEAR: {
      std::vector<QM31> w = r.qm31s();
      air = std::make_unique<MlLinearAir>(w);
      break;
    }
    default:
      throw WireError("unknown air id", -1);
  }
  r.end();
  return air;
}

}  // namespace orc
