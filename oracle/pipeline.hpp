// ORACLE — test infrastructure only. The standalone circle commit workload
// (64 columns x 2^20 M31 rows at blowup 4) composed from reference primitives:
//   1. circleIFFT per column on canonicHalf(log_rows)      ntt/circle.zig:272-346
//   2. zero-pad A and B separately to 2^(log_rows+log_blowup-1) each; the
//      interleaved FFT basis of size 2^k is the 2^(k+b) basis restricted to
//      its low k index bits (ntt/circle.zig:6-17), so this is the same polynomial
//   3. circleFFT per column on canonicHalf(log_rows+log_blowup) circle.zig:195-246
//   4. leaf r = hashM31s(row r of all columns), natural point order  m31/hash.zig:15-25
//   5. MerkleTree over the leaves                           core/merkle/merkle.zig:17-45
//   6. g[r] = sum_c gamma_c * LDE_c[r]  (QM31 x embedded M31)
//   7. n_folds FRI folds of g on the fri.zig domains of log size
//      log_rows+log_blowup with given alphas, each layer committed first
//      (hashQM31 leaves + tree) as in fri.zig:195-220.
#pragma once
#include <vector>

#include "circle.hpp"
#include "fri.hpp"

namespace orc {

// Root of the Merkle tree over `leaves` (merkle.zig:37-42), levels built in parallel.
inline Digest merkleRootParallel(std::vector<Digest> level, int threads) {
  while (level.size() > 1) {
    std::vector<Digest> up(level.size() / 2);
#pragma omp parallel for num_threads(threads) schedule(static)
    for (long i = 0; i < (long)up.size(); ++i) up[i] = hash2(level[2 * i], level[2 * i + 1]);
    level = std::move(up);
  }
  return level[0];
}

struct CommitResult {
  Digest lde_root;
  std::vector<Digest> layer_roots;
  std::vector<QM31> final_layer;
  std::vector<std::vector<M31>> lde;  // filled when keep_lde
  std::vector<QM31> g;                // filled when keep_lde
};

// `faithful` recomputes the twiddle tree inside every transform call exactly as
// the reference does (per-point coset.at()); otherwise one tree per domain.
inline CommitResult circleCommit(const std::vector<std::vector<M31>>& cols, unsigned log_rows,
                                 unsigned log_blowup, const std::vector<QM31>& gammas,
                                 const std::vector<QM31>& alphas, bool faithful, bool keep_lde,
                                 int threads) {
  const size_t C = cols.size();
  const unsigned log_N = log_rows + log_blowup;
  const size_t n = (size_t)1 << log_rows, N = (size_t)1 << log_N;
  CircleCoset small = CircleCoset::canonicHalf(log_rows);
  CircleCoset big = CircleCoset::canonicHalf(log_N);
  std::vector<M31> tw_small, tw_big;
  if (!faithful) {
    if (log_rows >= 3) tw_small = precomputeTwiddles(small, false);
    if (log_N >= 3) tw_big = precomputeTwiddles(big, false);
  }
  std::vector<std::vector<M31>> lde(C);
#pragma omp parallel for num_threads(threads) schedule(dynamic)
  for (long c = 0; c < (long)C; ++c) {
    std::vector<M31> coeffs = circleIFFT(cols[c], small, faithful || log_rows < 3 ? nullptr : &tw_small, faithful);
    std::vector<M31> padded(N, M31::zero());
    for (size_t i = 0; i < n / 2; ++i) {
      padded[i] = coeffs[i];
      padded[N / 2 + i] = coeffs[n / 2 + i];
    }
    lde[c] = circleFFT(padded, big, faithful || log_N < 3 ? nullptr : &tw_big, faithful);
  }
  std::vector<Digest> leaves(N);
  std::vector<QM31> g(N);
#pragma omp parallel for num_threads(threads) schedule(static)
  for (long r = 0; r < (long)N; ++r) {
    std::vector<M31> row(C);
    QM31 acc = QM31::zero();
    for (size_t c = 0; c < C; ++c) {
      row[c] = lde[c][r];
      acc = acc.add(gammas[c].mul(QM31::fromM31(row[c])));
    }
    leaves[r] = hashM31s(row.data(), C);
    g[r] = acc;
  }
  CommitResult res;
  res.lde_root = merkleRootParallel(leaves, threads);
  FriParams fp;  // only the domain log size matters for the layer domains
  fp.log_size = (uint8_t)log_N;
  fp.log_blowup = 0;
  std::vector<QM31> cur = g;
  QM31 it = invTwo();
  for (size_t i = 0; i < alphas.size(); ++i) {
    size_t ni = cur.size(), nn = ni / 2;
    std::vector<Digest> lv(ni);
#pragma omp parallel for num_threads(threads) schedule(static)
    for (long j = 0; j < (long)ni; ++j) lv[j] = hashQM31(cur[j]);
    res.layer_roots.push_back(merkleRootParallel(std::move(lv), threads));
    std::vector<QM31> dom = friDomainPoints(fp, (unsigned)i);
    std::vector<QM31> next(nn);
#pragma omp parallel for num_threads(threads) schedule(static)
    for (long j = 0; j < (long)nn; ++j) {
      QM31 y0 = cur[j], y1 = cur[j + nn];
      QM31 hs = y0.add(y1).mul(it);
      QM31 hd = y0.sub(y1).mul(dom[j].inv()).mul(it);
      next[j] = hs.add(alphas[i].mul(hd));
    }
    cur = std::move(next);
  }
  res.final_layer = cur;
  if (keep_lde) {
    res.lde = std::move(lde);
    res.g = std::move(g);
  }
  return res;
}

}  // namespace orc
