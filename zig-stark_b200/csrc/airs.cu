// Host-side AIR construction: public-input parsing, boundary assertions and the
// row-dependent constant polynomials of the two example AIRs.
#include "airs.cuh"
#include "host.cuh"

namespace zs {

namespace {

std::vector<qm31> subgroup_points(unsigned log_n) {
  const qm31 w = q_root_of_unity(log_n);
  std::vector<qm31> h(1u << log_n);
  qm31 acc = qone();
  for (auto& v : h) {
    v = acc;
    acc = qmul(acc, w);
  }
  return h;
}

// examples/rescue/src/main.zig:28-38: LCG round constants, top 31 bits, fromInt.
void rescue_round_constants(qm31 rc[7][4]) {
  uint64_t seed = 0x243f6a8885a308d3ull;
  for (int r = 0; r < 7; ++r)
    for (int j = 0; j < 4; ++j) {
      seed = seed * 6364136223846793005ull + 1442695040888963407ull;
      uint32_t v = (uint32_t)(seed >> 33);
      rc[r][j] = qfrom_m31(v >= P ? v % P : v);
    }
}

}  // namespace

void AirInfo::boundary(uint64_t n, std::vector<Boundary>& out) const {
  out.clear();
  switch (id) {
    case AIR_FIB:  // stark.zig:900-904
      out.push_back({0, 0, qzero()});
      out.push_back({1, 0, qone()});
      out.push_back({0, n - 1, pi[0]});
      break;
    case AIR_SEEDED_FIB:  // a_0, a_1 from the public inputs
      out.push_back({0, 0, pi[0]});
      out.push_back({1, 0, pi[1]});
      out.push_back({0, n - 1, pi[2]});
      break;
    case AIR_RESCUE_EXAMPLE:  // main.zig:125-130
    case AIR_RESCUE_STACKED:  // first permutation's input, last permutation's output
      for (uint32_t j = 0; j < 4; ++j) out.push_back({j, 0, pi[j]});
      for (uint32_t j = 0; j < 4; ++j) out.push_back({j, n - 1, pi[4 + j]});
      break;
    case AIR_LINEAR_EXAMPLE:  // main.zig:89-93: acc[0] = w_0 * x_0, acc[n-1] = claimed_y
      out.push_back({0, 0, qmul_m(x_inputs[0], 1)});
      out.push_back({0, n - 1, pi[0]});
      break;
    case AIR_ML_LINEAR:  // the last row, which the transitions leave unchecked, is a table row
      out.push_back({kMlSel, n - 1, qzero()});
      break;
    default:
      break;
  }
}

AirInfo make_air(uint32_t air_id, const uint8_t* pi_bytes, size_t pi_len) {
  AirInfo a;
  a.id = air_id;
  a.consts.id = air_id;
  WireReader r(pi_bytes, pi_len);
  switch (air_id) {
    case AIR_FIB:
      a.m = 2, a.num_trans = 2, a.num_bound = 3;
      a.pi.push_back(r.q());
      break;
    case AIR_SEEDED_FIB:
      a.m = 2, a.num_trans = 2, a.num_bound = 3;
      for (int i = 0; i < 3; ++i) a.pi.push_back(r.q());
      break;
    case AIR_RANGE_CHECK:  // stark.zig:964-974
    case AIR_MULTIPLICITY:  // stark.zig:1139-1149
      a.m = 3, a.n_pre = 1, a.n_lc = 1, a.n_rel = 1;
      a.sel[0] = 2, a.mult[0] = 1, a.n_keys[0] = 1, a.keys[0][0] = 0, a.tabs[0][0] = 0;
      break;
    case AIR_AND_TABLE:  // stark.zig:1048-1058
      a.m = 3, a.n_pre = 2, a.n_lc = 2, a.n_rel = 1;
      a.sel[0] = 2, a.mult[0] = 2, a.n_keys[0] = 2;
      a.keys[0][0] = 0, a.keys[0][1] = 1, a.tabs[0][0] = 0, a.tabs[0][1] = 1;
      break;
    case AIR_RESCUE_EXAMPLE: {  // examples/rescue/src/main.zig:69-144
      a.m = 4, a.num_trans = 4, a.num_bound = 8, a.fixed_n = 8, a.dc_mul = 5;
      for (int i = 0; i < 8; ++i) a.pi.push_back(r.q());
      qm31 rc[7][4];
      rescue_round_constants(rc);
      const std::vector<qm31> h = subgroup_points(3);
      a.consts.poly_len = 8;
      for (int j = 0; j < 4; ++j) {
        std::vector<qm31> ys(8);
        for (int k = 0; k < 8; ++k) ys[k] = k < 7 ? rc[k][j] : qzero();
        const std::vector<qm31> c = interpolate_small(h, ys);
        for (int k = 0; k < 8; ++k) a.consts.poly[j][k] = c[k];
      }
      break;
    }
    case AIR_RESCUE_STACKED: {
      a.m = 12, a.num_trans = 12, a.num_bound = 8, a.dc_mul = 2, a.dc_plus_n8 = true;
      for (int i = 0; i < 8; ++i) a.pi.push_back(r.q());
      qm31 rc[7][4];
      rescue_round_constants(rc);
      const std::vector<qm31> h = subgroup_points(3);
      a.consts.w8_7 = h[7];
      a.consts.poly_len = 8;
      for (int j = 0; j < 4; ++j) {
        std::vector<qm31> ys(8);
        for (int k = 0; k < 8; ++k) ys[k] = k < 7 ? rc[k][j] : qzero();
        const std::vector<qm31> c = interpolate_small(h, ys);
        for (int k = 0; k < 8; ++k) a.consts.poly[j][k] = c[k];
      }
      break;
    }
    case AIR_LINEAR_EXAMPLE: {  // examples/ml_linear/src/main.zig:21-116
      a.m = 1, a.num_trans = 1, a.num_bound = 2, a.fixed_n = 8;
      const uint64_t nx = r.len(16);
      for (uint64_t i = 0; i < nx; ++i) a.x_inputs.push_back(r.q());
      a.pi.push_back(r.q());
      if (a.x_inputs.size() != 8) throw Error(ZS_EMALFORMED, "linear example AIR takes 8 inputs");
      const std::vector<qm31> h = subgroup_points(3);
      std::vector<qm31> ys(8);
      for (int k = 0; k < 8; ++k) ys[k] = qmul_m(a.x_inputs[(k + 1) % 8], (uint32_t)((k + 1) % 8 + 1));
      const std::vector<qm31> c = interpolate_small(h, ys);
      a.consts.poly_len = 8;
      for (int k = 0; k < 8; ++k) a.consts.poly[0][k] = c[k];
      break;
    }
    case AIR_ML_LINEAR: {
      a.m = kMlCols, a.n_pre = kMlDim, a.n_lc = kMlDim, a.n_rel = 1, a.num_trans = kMlDim, a.num_bound = 1;
      a.sel[0] = kMlSel, a.mult[0] = kMlMult;  // keys x_l and table columns P_l, l < kMlDim (implicit)
      const uint64_t nw = r.len(16);
      if (nw != (uint64_t)kMlDim * kMlDim) throw Error(ZS_EMALFORMED, "linear layer AIR takes a 128 x 128 matrix");
      a.w.resize(nw);
      for (uint64_t k = 0; k < nw; ++k) {
        const qm31 v = r.q();
        if (v.a.b || v.b.a || v.b.b) throw Error(ZS_EMALFORMED, "linear layer weights are M31 values");
        a.w[k] = v.a.a;
      }
      break;
    }
    default:
      throw Error(ZS_EGENERIC, "unknown AIR id");
  }
  r.end();
  return a;
}

}  // namespace zs
