// ORACLE — test infrastructure only. C entry points over the CPU restatement,
// loaded by the tests (ctypes) as the checker for the GPU backend. Buffers the
// oracle returns are malloc'ed and released with orc_free.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <vector>

#include "binius.hpp"
#include "pipeline.hpp"
#include "stark.hpp"

using namespace orc;

namespace {
uint8_t* dupBytes(const std::vector<uint8_t>& v, size_t* out_len) {
  uint8_t* p = (uint8_t*)std::malloc(v.empty() ? 1 : v.size());
  if (!v.empty()) std::memcpy(p, v.data(), v.size());
  *out_len = v.size();
  return p;
}
QM31 q4(const uint32_t* w) { return QM31::make(w[0], w[1], w[2], w[3]); }
void put4(const QM31& v, uint32_t* w) {
  w[0] = v.a.c0.v;
  w[1] = v.a.c1.v;
  w[2] = v.b.c0.v;
  w[3] = v.b.c1.v;
}
}  // namespace

extern "C" {

void orc_free(void* p) { std::free(p); }

void orc_blake3(const uint8_t* msg, size_t len, uint8_t* out32) { blake3Hash(msg, len, out32); }

void orc_hash2(const uint8_t* a, const uint8_t* b, uint8_t* out32) {
  Digest x, y;
  std::memcpy(x.data(), a, 32);
  std::memcpy(y.data(), b, 32);
  Digest d = hash2(x, y);
  std::memcpy(out32, d.data(), 32);
}

void orc_hash_qm31(const uint32_t* v, size_t n, uint8_t* out) {
  for (size_t i = 0; i < n; ++i) {
    Digest d = hashQM31(q4(v + 4 * i));
    std::memcpy(out + 32 * i, d.data(), 32);
  }
}

// Row leaves: values laid out row-major (n_rows x n_cols).
void orc_hash_m31_rows(const uint32_t* v, size_t n_rows, size_t n_cols, uint8_t* out) {
  std::vector<M31> row(n_cols);
  for (size_t r = 0; r < n_rows; ++r) {
    for (size_t c = 0; c < n_cols; ++c) row[c] = M31(v[r * n_cols + c]);
    Digest d = hashM31s(row.data(), n_cols);
    std::memcpy(out + 32 * r, d.data(), 32);
  }
}

// op: 0 add, 1 sub, 2 mul, 3 neg, 4 inv
void orc_m31_op(int op, const uint32_t* a, const uint32_t* b, uint32_t* out, size_t n) {
  for (size_t i = 0; i < n; ++i) {
    M31 x(a[i]), y(b ? b[i] : 0);
    M31 r;
    switch (op) {
      case 0: r = x.add(y); break;
      case 1: r = x.sub(y); break;
      case 2: r = x.mul(y); break;
      case 3: r = x.neg(); break;
      default: r = x.inv(); break;
    }
    out[i] = r.v;
  }
}

void orc_qm31_op(int op, const uint32_t* a, const uint32_t* b, uint32_t* out, size_t n) {
  for (size_t i = 0; i < n; ++i) {
    QM31 x = q4(a + 4 * i), y = b ? q4(b + 4 * i) : QM31::zero();
    QM31 r;
    switch (op) {
      case 0: r = x.add(y); break;
      case 1: r = x.sub(y); break;
      case 2: r = x.mul(y); break;
      case 3: r = x.neg(); break;
      default: r = x.inv(); break;
    }
    put4(r, out + 4 * i);
  }
}

void orc_qm31_pow(const uint32_t* a, uint64_t e, uint32_t* out) { put4(q4(a).pow(e), out); }
void orc_qm31_root(unsigned log_size, uint32_t* out) { put4(QM31::primitiveRootOfUnity(log_size), out); }

void orc_circle_generator_mul(uint64_t scalar, uint32_t* out_xy) {
  CirclePoint p = CirclePoint::generator().mulScalar(scalar);
  out_xy[0] = p.x.v;
  out_xy[1] = p.y.v;
}

// Natural-order points of the domain canonicHalf(log_n) ++ conjugate.
void orc_circle_domain(unsigned log_n, uint32_t* xs, uint32_t* ys) {
  CircleCoset hc = CircleCoset::canonicHalf(log_n);
  size_t n = (size_t)1 << log_n;
  for (size_t i = 0; i < n; ++i) {
    CirclePoint p = circleDomainPoint(hc, i);
    xs[i] = p.x.v;
    ys[i] = p.y.v;
  }
}

// circleFFT / circleIFFT on canonicHalf(log_n); coefficients A-then-B.
void orc_circle_fft(const uint32_t* coeffs, unsigned log_n, uint32_t* evals, int faithful) {
  size_t n = (size_t)1 << log_n;
  std::vector<M31> c(n);
  for (size_t i = 0; i < n; ++i) c[i] = M31(coeffs[i]);
  std::vector<M31> e = circleFFT(c, CircleCoset::canonicHalf(log_n), nullptr, faithful != 0);
  for (size_t i = 0; i < n; ++i) evals[i] = e[i].v;
}
void orc_circle_ifft(const uint32_t* evals, unsigned log_n, uint32_t* coeffs, int faithful) {
  size_t n = (size_t)1 << log_n;
  std::vector<M31> e(n);
  for (size_t i = 0; i < n; ++i) e[i] = M31(evals[i]);
  std::vector<M31> c = circleIFFT(e, CircleCoset::canonicHalf(log_n), nullptr, faithful != 0);
  for (size_t i = 0; i < n; ++i) coeffs[i] = c[i].v;
}
uint32_t orc_circle_eval_at(const uint32_t* coeffs, unsigned log_n, uint32_t x, uint32_t y) {
  size_t n = (size_t)1 << log_n;
  std::vector<M31> c(n);
  for (size_t i = 0; i < n; ++i) c[i] = M31(coeffs[i]);
  return circleEvalAtPoint(c, CirclePoint(M31(x), M31(y))).v;
}
// The twiddle tree of canonicHalf(log_n) (length 2^(log_n-1)), as circle.zig:69-82 builds it.
void orc_circle_twiddles(unsigned log_n, uint32_t* out) {
  std::vector<M31> t = precomputeTwiddles(CircleCoset::canonicHalf(log_n), false);
  for (size_t i = 0; i < t.size(); ++i) out[i] = t[i].v;
}

// Merkle root over 32-byte leaves; optionally the full opening path of `index`.
void orc_merkle_root(const uint8_t* leaves, size_t n, uint8_t* out32) {
  std::vector<Digest> l(n);
  for (size_t i = 0; i < n; ++i) std::memcpy(l[i].data(), leaves + 32 * i, 32);
  MerkleTree t(l);
  std::memcpy(out32, t.root().data(), 32);
}

// Interpolation (O(n^2) reference algorithm or NTT) on H = <w_n>, n = 2^log_n.
void orc_interpolate_subgroup(const uint32_t* ys, unsigned log_n, int use_ntt, uint32_t* coeffs) {
  size_t n = (size_t)1 << log_n;
  std::vector<QM31> y(n);
  for (size_t i = 0; i < n; ++i) y[i] = q4(ys + 4 * i);
  std::vector<QM31> c;
  if (use_ntt) {
    c = interpolateSubgroupNtt(y, log_n);
  } else {
    std::vector<QM31> xs(n);
    QM31 w = QM31::primitiveRootOfUnity(log_n), acc = QM31::one();
    for (size_t i = 0; i < n; ++i) {
      xs[i] = acc;
      acc = acc.mul(w);
    }
    c = interpolateLagrange(xs, y);
  }
  for (size_t i = 0; i < n; ++i) put4(c[i], coeffs + 4 * i);
}

// Evaluations of `coeffs` on FRI_OFFSET * <w_N> (Horner or NTT).
void orc_evaluate_coset(const uint32_t* coeffs, size_t n, unsigned log_N, int use_ntt, uint32_t* out) {
  std::vector<QM31> c(n);
  for (size_t i = 0; i < n; ++i) c[i] = q4(coeffs + 4 * i);
  size_t N = (size_t)1 << log_N;
  std::vector<QM31> e;
  if (use_ntt) {
    e = evaluateCosetNtt(c, friOffset(), log_N);
  } else {
    e.resize(N);
    QM31 w = QM31::primitiveRootOfUnity(log_N), d = friOffset();
    for (size_t i = 0; i < N; ++i) {
      e[i] = evalHorner(c, d);
      d = d.mul(w);
    }
  }
  for (size_t i = 0; i < N; ++i) put4(e[i], out + 4 * i);
}

// Channel script: absorbs `absorb` (raw bytes), then samples n_qm31 QM31 words
// followed by n_idx indices below `idx_bound`.
void orc_channel_script(const uint8_t* sep, size_t sep_len, const uint8_t* absorb, size_t absorb_len,
                        size_t n_qm31, uint32_t* out_qm31, size_t n_idx, uint64_t idx_bound,
                        uint64_t* out_idx) {
  Channel ch(sep, sep_len);
  ch.absorbBytes(absorb, absorb_len);
  for (size_t i = 0; i < n_qm31; ++i) put4(ch.sampleQM31(), out_qm31 + 4 * i);
  for (size_t i = 0; i < n_idx; ++i) out_idx[i] = ch.sampleIndex(idx_bound);
}

// FRI prove over an explicit codeword; returns the serialized Fri.Proof.
int orc_fri_prove_codeword(uint8_t log_size, uint8_t log_blowup, uint64_t num_queries,
                           uint8_t remainder_log, const uint32_t* codeword, const uint8_t* sep,
                           size_t sep_len, uint8_t** out, size_t* out_len) {
  try {
    FriParams p;
    p.log_size = log_size;
    p.log_blowup = log_blowup;
    p.num_queries = num_queries;
    p.remainder_log = remainder_log;
    size_t n0 = (size_t)1 << p.domainLogSize();
    std::vector<QM31> cw(n0);
    for (size_t i = 0; i < n0; ++i) cw[i] = q4(codeword + 4 * i);
    Channel ch(sep, sep_len);
    FriProof f = friProveCodeword(p, cw, ch);
    Writer w;
    f.write(w);
    *out = dupBytes(w.out, out_len);
    return 0;
  } catch (const WireError& e) {
    return e.code;
  } catch (...) {
    return -1;
  }
}

int orc_fri_verify(uint8_t log_size, uint8_t log_blowup, uint64_t num_queries, uint8_t remainder_log,
                   const uint8_t* proof, size_t proof_len, const uint8_t* sep, size_t sep_len, int* ok) {
  try {
    FriParams p;
    p.log_size = log_size;
    p.log_blowup = log_blowup;
    p.num_queries = num_queries;
    p.remainder_log = remainder_log;
    Reader r(proof, proof_len);
    FriProof f = FriProof::read(r);
    r.end();
    Channel ch(sep, sep_len);
    *ok = friVerify(p, f, ch) ? 1 : 0;
    return 0;
  } catch (const WireError& e) {
    return e.code;
  } catch (...) {
    return -1;
  }
}

// GenericStark(Air).proveWithPreprocessed. params: wire StarkParams; columns in
// wire form []const []const QM31; mode 0 = reference interpolation, 1 = NTT.
int orc_prove(uint32_t air_id, const uint8_t* params, size_t params_len, const uint8_t* pi,
              size_t pi_len, const uint8_t* pre, size_t pre_len, const uint8_t* trace,
              size_t trace_len, const uint8_t* sep, size_t sep_len, int mode, uint8_t** out,
              size_t* out_len) {
  try {
    Reader pr(params, params_len);
    StarkParams sp = StarkParams::read(pr);
    pr.end();
    auto air = makeAir(air_id, pi, pi_len);
    auto pcols = readColumns(pre, pre_len);
    auto tcols = readColumns(trace, trace_len);
    Stark st(*air);
    Channel ch(sep, sep_len);
    StarkProof proof = st.prove(sp, pcols, tcols, ch, mode ? Mode::Ntt : Mode::Lagrange);
    *out = dupBytes(proof.serialize(), out_len);
    return 0;
  } catch (const WireError& e) {
    return e.code;
  } catch (const std::bad_alloc&) {
    return -3;
  } catch (...) {
    return -1;
  }
}

int orc_verify(uint32_t air_id, const uint8_t* params, size_t params_len, const uint8_t* pi,
               size_t pi_len, const uint8_t* proof, size_t proof_len, const uint8_t* sep,
               size_t sep_len, int* ok) {
  try {
    Reader pr(params, params_len);
    StarkParams sp = StarkParams::read(pr);
    pr.end();
    auto air = makeAir(air_id, pi, pi_len);
    StarkProof p = StarkProof::deserialize(proof, proof_len);
    Stark st(*air);
    Channel ch(sep, sep_len);
    *ok = st.verify(sp, p, ch) ? 1 : 0;
    return 0;
  } catch (const WireError& e) {
    return e.code;
  } catch (...) {
    return -1;
  }
}

// Per-column commitment roots (stark.zig:397-414): NTT interpolation on H, coset
// evaluation on D, MerkleTree over hashQM31 leaves. out: 32 bytes per column.
int orc_commit_columns(const uint8_t* cols, size_t cols_len, unsigned trace_log, unsigned log_blowup, uint8_t* out) {
  try {
    auto c = readColumns(cols, cols_len);
    for (size_t j = 0; j < c.size(); ++j) {
      std::vector<QM31> coeffs = interpolateSubgroupNtt(c[j], trace_log);
      std::vector<QM31> cw = evaluateCosetNtt(coeffs, friOffset(), trace_log + log_blowup);
      MerkleTree t(hashCodeword(cw));
      std::memcpy(out + 32 * j, t.root().data(), 32);
    }
    return 0;
  } catch (const WireError& e) {
    return e.code;
  } catch (...) {
    return -1;
  }
}

// Re-serializes a proof after a round trip through the wire reader.
// Binius tower multiply at `level` (1..7) of two little-endian u128 values (2 x u64).
void orc_tower_mul(unsigned level, const uint64_t* a, const uint64_t* b, uint64_t* out) {
  const u128 x = ((u128)a[1] << 64) | a[0], y = ((u128)b[1] << 64) | b[0];
  const u128 r = towerMul(level, x & towerMask(level), y & towerMask(level));
  out[0] = (uint64_t)r;
  out[1] = (uint64_t)(r >> 64);
}

// One sum-check round's values[t] in the flattened form of the accelerator hook
// (src/binius/accel.zig:9-26, 43-47): level 3 (Gf256, one byte per element) or level 7
// (Gf2_128, 16 little-endian bytes per element). Returns 0, or -2 on malformed input.
int orc_binius_values(unsigned level, const uint8_t* cur_flat, size_t len, size_t m, const uint8_t* coeffs,
                      size_t nterms, const uint32_t* indices, size_t n_indices, const uint32_t* offsets,
                      size_t dmax, size_t half, uint8_t* out) {
  if (level != 3 && level != 7) return -2;
  const size_t es = level == 3 ? 1 : 16;
  if (2 * half > len || offsets[0] != 0 || offsets[nterms] != n_indices) return -2;
  auto get = [&](const uint8_t* p) {
    u128 v = 0;
    for (size_t k = 0; k < es; ++k) v |= (u128)p[k] << (8 * k);
    return v;
  };
  std::vector<std::vector<u128>> cur(m, std::vector<u128>(len));
  for (size_t f = 0; f < m; ++f)
    for (size_t i = 0; i < len; ++i) cur[f][i] = get(cur_flat + (f * len + i) * es);
  std::vector<u128> cf(nterms);
  for (size_t k = 0; k < nterms; ++k) cf[k] = get(coeffs + k * es);
  for (size_t j = 0; j < n_indices; ++j)
    if (indices[j] >= m) return -2;
  const std::vector<uint32_t> idx(indices, indices + n_indices), off(offsets, offsets + nterms + 1);
  const std::vector<u128> v = sumcheckRoundValues(level, cur, cf, idx, off, dmax, half);
  for (size_t t = 0; t <= dmax; ++t)
    for (size_t k = 0; k < es; ++k) out[t * es + k] = (uint8_t)(v[t] >> (8 * k));
  return 0;
}

// SHA-256 of msg (the transcript hash of src/binius/sumcheck.zig:47-87).
void orc_sha256(const uint8_t* msg, size_t n, uint8_t* out) {
  const auto h = sha256(msg, n);
  std::memcpy(out, h.data(), 32);
}

namespace {
bool binius_inputs(unsigned level, const uint8_t* tables, size_t len, size_t m, const uint8_t* coeffs, size_t nterms,
                   const uint32_t* indices, size_t n_indices, const uint32_t* offsets,
                   std::vector<std::vector<u128>>& cur, SumcheckTerms& tm) {
  if (level != 3 && level != 7) return false;
  if (offsets[0] != 0 || offsets[nterms] != n_indices) return false;
  for (size_t j = 0; j < n_indices; ++j)
    if (indices[j] >= m) return false;
  const size_t es = towerSize(level);
  cur.assign(m, std::vector<u128>(len));
  for (size_t f = 0; f < m; ++f)
    for (size_t i = 0; i < len; ++i) cur[f][i] = towerFromBytes(level, tables + (f * len + i) * es);
  tm.coeffs.resize(nterms);
  for (size_t k = 0; k < nterms; ++k) tm.coeffs[k] = towerFromBytes(level, coeffs + k * es);
  tm.indices.assign(indices, indices + n_indices);
  tm.offsets.assign(offsets, offsets + nterms + 1);
  return true;
}
}  // namespace

// Sumcheck(F).proveCombination (with its optional transcript seed when has_seed): claimed_out one
// element, rounds_out k * (dmax + 1) elements.
int orc_binius_prove(unsigned level, const uint8_t* tables, size_t k, size_t m, const uint8_t* coeffs, size_t nterms,
                     const uint32_t* indices, size_t n_indices, const uint32_t* offsets, const uint8_t* seed,
                     size_t seed_len, int has_seed, uint8_t* claimed_out, uint8_t* rounds_out) {
  std::vector<std::vector<u128>> cur;
  SumcheckTerms tm;
  if (!binius_inputs(level, tables, (size_t)1 << k, m, coeffs, nterms, indices, n_indices, offsets, cur, tm)) return -2;
  const std::vector<uint8_t> sd(seed, seed + (has_seed ? seed_len : 0));
  const SumcheckProof pf = proveCombination(level, k, cur, tm, has_seed ? &sd : nullptr);
  const size_t es = towerSize(level), d1 = tm.dmax() + 1;
  towerToBytes(level, pf.claimed, claimed_out);
  for (size_t i = 0; i < k; ++i)
    for (size_t t = 0; t < d1; ++t) towerToBytes(level, pf.rounds[i][t], rounds_out + (i * d1 + t) * es);
  return 0;
}

// 1 when the proof replays and ends at g(challenges), 0 when not, -2 for bad inputs.
int orc_binius_verify(unsigned level, const uint8_t* tables, size_t k, size_t m, const uint8_t* coeffs, size_t nterms,
                      const uint32_t* indices, size_t n_indices, const uint32_t* offsets, const uint8_t* seed,
                      size_t seed_len, int has_seed, const uint8_t* claimed, const uint8_t* rounds) {
  std::vector<std::vector<u128>> cur;
  SumcheckTerms tm;
  if (!binius_inputs(level, tables, (size_t)1 << k, m, coeffs, nterms, indices, n_indices, offsets, cur, tm)) return -2;
  const size_t es = towerSize(level), d1 = tm.dmax() + 1;
  SumcheckProof pf{towerFromBytes(level, claimed), std::vector<std::vector<u128>>(k, std::vector<u128>(d1))};
  for (size_t i = 0; i < k; ++i)
    for (size_t t = 0; t < d1; ++t) pf.rounds[i][t] = towerFromBytes(level, rounds + (i * d1 + t) * es);
  const std::vector<uint8_t> sd(seed, seed + (has_seed ? seed_len : 0));
  return verifyCombination(level, k, cur, tm, pf, has_seed ? &sd : nullptr) ? 1 : 0;
}

// The fold of m tables of len elements at r into m tables of len / 2 (next).
int orc_binius_fold(unsigned level, const uint8_t* tables, size_t len, size_t m, const uint8_t* r, uint8_t* next) {
  if (level != 3 && level != 7) return -2;
  const size_t es = towerSize(level);
  std::vector<std::vector<u128>> cur(m, std::vector<u128>(len));
  for (size_t f = 0; f < m; ++f)
    for (size_t i = 0; i < len; ++i) cur[f][i] = towerFromBytes(level, tables + (f * len + i) * es);
  foldTables(level, cur, len, towerFromBytes(level, r));
  for (size_t f = 0; f < m; ++f)
    for (size_t i = 0; i < len / 2; ++i) towerToBytes(level, cur[f][i], next + (f * (len / 2) + i) * es);
  return 0;
}

// A transcript seeded with `seed` absorbing one-element coefficient lists in turn
// (sumcheck.zig:697-713): out[i] = the challenge after absorbing element i.
int orc_binius_challenges(unsigned level, const uint8_t* seed, size_t seed_len, const uint8_t* elems, size_t n,
                          uint8_t* out) {
  if (level != 3 && level != 7) return -2;
  const size_t es = towerSize(level);
  SumcheckTranscript tr = SumcheckTranscript::initBytes(level, std::vector<uint8_t>(seed, seed + seed_len));
  for (size_t i = 0; i < n; ++i) towerToBytes(level, tr.absorb({towerFromBytes(level, elems + i * es)}), out + i * es);
  return 0;
}

// interpolateCoeffs through the points 0..n-1 (n <= 64).
int orc_binius_interpolate(unsigned level, const uint8_t* values, size_t n, uint8_t* coeffs_out) {
  if ((level != 3 && level != 7) || n == 0 || n > 64) return -2;
  const size_t es = towerSize(level);
  std::vector<u128> pts(n), vals(n);
  for (size_t i = 0; i < n; ++i) {
    pts[i] = (u128)i;
    vals[i] = towerFromBytes(level, values + i * es);
  }
  const std::vector<u128> cs = interpolateCoeffs(level, pts, vals);
  for (size_t i = 0; i < n; ++i) towerToBytes(level, cs[i], coeffs_out + i * es);
  return 0;
}

// serialization.zig:220-250 "golden wire layout is stable": the struct
// {name: [3]u8 = "abc", count: u32 = 0x01020304, rows: []u16 = {0x0102, 0x0304},
// flag: bool = true, maybe: ?[2]u8 = {0xde, 0xad}} through the oracle's Writer.
// Writes at most 64 bytes; returns the length.
size_t orc_wire_golden(uint8_t* out) {
  Writer w;
  const uint8_t name[3] = {'a', 'b', 'c'};
  w.raw(name, 3);
  w.uint_le(0x01020304u, 4);
  const uint16_t rows[2] = {0x0102, 0x0304};
  w.u64(2);
  for (uint16_t r : rows) w.uint_le(r, 2);
  w.flag(true);
  const uint8_t maybe[2] = {0xde, 0xad};
  w.flag(true);
  w.raw(maybe, 2);
  std::memcpy(out, w.out.data(), std::min<size_t>(w.out.size(), 64));
  return w.out.size();
}

int orc_proof_roundtrip(const uint8_t* proof, size_t proof_len, uint8_t** out, size_t* out_len) {
  try {
    StarkProof p = StarkProof::deserialize(proof, proof_len);
    *out = dupBytes(p.serialize(), out_len);
    return 0;
  } catch (const WireError& e) {
    return e.code;
  } catch (...) {
    return -1;
  }
}

// The circle commit workload. trace: n_cols x 2^log_rows column-major.
// gammas: n_cols QM31, alphas: n_folds QM31. Outputs: lde_root (32 B),
// layer_roots (32 B x n_folds), final_layer (QM31 x 2^(log_rows+log_blowup-n_folds)),
// optional lde (n_cols x 2^(log_rows+log_blowup)) and g (QM31 x 2^(...)).
int orc_circle_commit(const uint32_t* trace, uint32_t n_cols, uint32_t log_rows, uint32_t log_blowup,
                      const uint32_t* gammas, const uint32_t* alphas, uint32_t n_folds, int faithful,
                      int threads, uint8_t* lde_root, uint8_t* layer_roots, uint32_t* final_layer,
                      uint32_t* lde_out, uint32_t* g_out) {
  try {
    size_t n = (size_t)1 << log_rows;
    std::vector<std::vector<M31>> cols(n_cols, std::vector<M31>(n));
    for (size_t c = 0; c < n_cols; ++c)
      for (size_t i = 0; i < n; ++i) cols[c][i] = M31(trace[c * n + i]);
    std::vector<QM31> gs(n_cols), as(n_folds);
    for (size_t c = 0; c < n_cols; ++c) gs[c] = q4(gammas + 4 * c);
    for (size_t i = 0; i < n_folds; ++i) as[i] = q4(alphas + 4 * i);
    CommitResult r = circleCommit(cols, log_rows, log_blowup, gs, as, faithful != 0,
                                  lde_out != nullptr || g_out != nullptr, threads);
    std::memcpy(lde_root, r.lde_root.data(), 32);
    for (size_t i = 0; i < r.layer_roots.size(); ++i) std::memcpy(layer_roots + 32 * i, r.layer_roots[i].data(), 32);
    for (size_t i = 0; i < r.final_layer.size(); ++i) put4(r.final_layer[i], final_layer + 4 * i);
    size_t N = (size_t)1 << (log_rows + log_blowup);
    if (lde_out)
      for (size_t c = 0; c < n_cols; ++c)
        for (size_t i = 0; i < N; ++i) lde_out[c * N + i] = r.lde[c][i].v;
    if (g_out)
      for (size_t i = 0; i < N; ++i) put4(r.g[i], g_out + 4 * i);
    return 0;
  } catch (...) {
    return -1;
  }
}

}  // extern "C"
