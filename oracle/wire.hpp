// ORACLE — test infrastructure only. Proof structures and the canonical wire
// encoding, restated from src/core/serialization.zig:58-190 and docs/wire.md:
// little-endian ints, usize as 8 bytes, slices as u64 length + elements,
// optionals as a 1-byte flag, structs in declaration order, allocator fields
// skipped, field elements as SIZE LE bytes.
#pragma once
#include <cstdint>
#include <optional>
#include <stdexcept>
#include <string>
#include <vector>

#include "hash.hpp"

namespace orc {

struct WireError : std::runtime_error {
  int code;
  WireError(const char* m, int c) : std::runtime_error(m), code(c) {}
};

struct Writer {
  std::vector<uint8_t> out;
  // serialization.zig:58-120: ints little-endian at their own width, usize and slice
  // lengths as u64, bool and an optional's presence as one byte, arrays raw.
  void uint_le(uint64_t v, unsigned width) {
    for (unsigned i = 0; i < width; ++i) out.push_back((uint8_t)(v >> (8 * i)));
  }
  void u8(uint8_t v) { uint_le(v, 1); }
  void u64(uint64_t v) { uint_le(v, 8); }
  void flag(bool present) { u8(present ? 1 : 0); }
  void raw(const uint8_t* p, size_t n) { out.insert(out.end(), p, p + n); }
  void digest(const Digest& d) { out.insert(out.end(), d.begin(), d.end()); }
  void qm31(const QM31& v) {
    uint8_t b[16];
    v.toBytes(b);
    out.insert(out.end(), b, b + 16);
  }
  void digests(const std::vector<Digest>& v) {
    u64(v.size());
    for (auto& d : v) digest(d);
  }
  void qm31s(const std::vector<QM31>& v) {
    u64(v.size());
    for (auto& x : v) qm31(x);
  }
};

struct Reader {
  const uint8_t* p;
  size_t n, pos = 0;
  Reader(const uint8_t* d, size_t len) : p(d), n(len) {}
  const uint8_t* take(size_t k) {
    if (pos + k > n || pos + k < pos) throw WireError("unexpected end", -2);
    const uint8_t* r = p + pos;
    pos += k;
    return r;
  }
  uint8_t u8() { return *take(1); }
  uint64_t u64() {
    const uint8_t* b = take(8);
    uint64_t v = 0;
    for (int i = 0; i < 8; ++i) v |= (uint64_t)b[i] << (8 * i);
    return v;
  }
  uint64_t len() {
    uint64_t l = u64();
    if (l > n) throw WireError("length prefix exceeds input", -2);
    return l;
  }
  Digest digest() {
    Digest d;
    const uint8_t* b = take(32);
    std::copy(b, b + 32, d.begin());
    return d;
  }
  QM31 qm31() { return QM31::fromBytes(take(16)); }
  std::vector<Digest> digests() {
    uint64_t l = len();
    std::vector<Digest> v;
    for (uint64_t i = 0; i < l; ++i) v.push_back(digest());
    return v;
  }
  std::vector<QM31> qm31s() {
    uint64_t l = len();
    std::vector<QM31> v;
    for (uint64_t i = 0; i < l; ++i) v.push_back(qm31());
    return v;
  }
  void end() {
    if (pos != n) throw WireError("trailing bytes", -2);
  }
};

// stark.zig:75-90.
struct StarkParams {
  uint8_t trace_log = 0;
  uint8_t log_blowup = 3;
  uint64_t num_queries = 16;
  uint8_t remainder_log = 3;
  size_t traceLen() const { return (size_t)1 << trace_log; }
  size_t domainLen() const { return (size_t)1 << (trace_log + log_blowup); }
  size_t shift() const { return (size_t)1 << log_blowup; }
  void write(Writer& w) const {
    w.u8(trace_log);
    w.u8(log_blowup);
    w.u64(num_queries);
    w.u8(remainder_log);
  }
  static StarkParams read(Reader& r) {
    StarkParams p;
    p.trace_log = r.u8();
    p.log_blowup = r.u8();
    p.num_queries = r.u64();
    p.remainder_log = r.u8();
    return p;
  }
};

// fri.zig:38-55.
struct FriParams {
  uint8_t log_size = 0;
  uint8_t log_blowup = 3;
  uint64_t num_queries = 24;
  uint8_t remainder_log = 3;
  unsigned domainLogSize() const { return log_size + log_blowup; }
  unsigned numFoldRounds() const { return domainLogSize() - remainder_log; }
  void write(Writer& w) const {
    w.u8(log_size);
    w.u8(log_blowup);
    w.u64(num_queries);
    w.u8(remainder_log);
  }
  static FriParams read(Reader& r) {
    FriParams p;
    p.log_size = r.u8();
    p.log_blowup = r.u8();
    p.num_queries = r.u64();
    p.remainder_log = r.u8();
    return p;
  }
};

// fri.zig:58-93.
struct FriPair {
  QM31 value0, value1;
  std::vector<Digest> path0, path1;
};
struct FriQuery {
  uint64_t index = 0;
  std::vector<FriPair> pairs;
};
struct FriProof {
  FriParams params;
  std::vector<Digest> roots;
  std::vector<QM31> remainder;
  std::vector<FriQuery> queries;
  void write(Writer& w) const {
    params.write(w);
    w.digests(roots);
    w.qm31s(remainder);
    w.u64(queries.size());
    for (auto& q : queries) {
      w.u64(q.index);
      w.u64(q.pairs.size());
      for (auto& p : q.pairs) {
        w.qm31(p.value0);
        w.qm31(p.value1);
        w.digests(p.path0);
        w.digests(p.path1);
      }
    }
  }
  static FriProof read(Reader& r) {
    FriProof f;
    f.params = FriParams::read(r);
    f.roots = r.digests();
    f.remainder = r.qm31s();
    uint64_t nq = r.len();
    for (uint64_t i = 0; i < nq; ++i) {
      FriQuery q;
      q.index = r.u64();
      uint64_t np = r.len();
      for (uint64_t k = 0; k < np; ++k) {
        FriPair p;
        p.value0 = r.qm31();
        p.value1 = r.qm31();
        p.path0 = r.digests();
        p.path1 = r.digests();
        q.pairs.push_back(std::move(p));
      }
      f.queries.push_back(std::move(q));
    }
    return f;
  }
};

// stark.zig:97-137.
struct QueryReveal {
  uint64_t query_index = 0;
  std::vector<QM31> values;
  std::vector<std::vector<Digest>> paths;
};
struct StarkProof {
  StarkParams params;
  std::vector<Digest> trace_roots;
  std::optional<std::vector<Digest>> preprocessed_roots;
  std::optional<std::vector<Digest>> accumulator_roots;
  Digest quotient_root{};
  std::vector<QM31> deep_evals;
  FriProof fri;
  std::vector<QueryReveal> queries;

  std::vector<uint8_t> serialize() const {
    Writer w;
    params.write(w);
    w.digests(trace_roots);
    if (preprocessed_roots) {
      w.u8(1);
      w.digests(*preprocessed_roots);
    } else {
      w.u8(0);
    }
    if (accumulator_roots) {
      w.u8(1);
      w.digests(*accumulator_roots);
    } else {
      w.u8(0);
    }
    w.digest(quotient_root);
    w.qm31s(deep_evals);
    fri.write(w);
    w.u64(queries.size());
    for (auto& q : queries) {
      w.u64(q.query_index);
      w.qm31s(q.values);
      w.u64(q.paths.size());
      for (auto& p : q.paths) w.digests(p);
    }
    return w.out;
  }
  static StarkProof deserialize(const uint8_t* d, size_t n) {
    Reader r(d, n);
    StarkProof s;
    s.params = StarkParams::read(r);
    s.trace_roots = r.digests();
    uint8_t f = r.u8();
    if (f == 1) s.preprocessed_roots = r.digests();
    f = r.u8();
    if (f == 1) s.accumulator_roots = r.digests();
    s.quotient_root = r.digest();
    s.deep_evals = r.qm31s();
    s.fri = FriProof::read(r);
    uint64_t nq = r.len();
    for (uint64_t i = 0; i < nq; ++i) {
      QueryReveal q;
      q.query_index = r.u64();
      q.values = r.qm31s();
      uint64_t np = r.len();
      for (uint64_t k = 0; k < np; ++k) q.paths.push_back(r.digests());
      s.queries.push_back(std::move(q));
    }
    r.end();
    return s;
  }
};

// Columns in wire form: []const []const QM31.
inline std::vector<std::vector<QM31>> readColumns(const uint8_t* d, size_t n) {
  std::vector<std::vector<QM31>> cols;
  if (n == 0) return cols;
  Reader r(d, n);
  uint64_t m = r.len();
  for (uint64_t j = 0; j < m; ++j) cols.push_back(r.qm31s());
  r.end();
  return cols;
}

}  // namespace orc
