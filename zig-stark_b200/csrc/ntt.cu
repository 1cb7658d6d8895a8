// NTTs over QM31 for the low-degree extension, computed in the CRT domain.
//
// QM31 = CM31[j]/(j^2 + i), and -i = s^2 with s = 2^15 (1 - i), so
//   phi: a + b j  ->  (a + b s, a - b s)
// is a ring isomorphism QM31 -> CM31 x CM31. Both components of the 2-adic root have
// order 2^32, so a DFT over a 2-power subgroup of QM31 is two CM31 DFTs with the
// component roots: every butterfly costs two CM31 products (3 M31 products each)
// instead of one QM31 product (9). phi and its inverse
//   a = (u + v) / 2,  b = (u - v) / (2 s) = (u - v)(1 + i) 2^-17
// are additions and rotations of the 31-bit word. The transform is exact, so its
// results equal the reference's Lagrange interpolation / Horner evaluation value for
// value (the DFT over the subgroup is invertible in both components).
//
// The LDE: the inverse transform on H runs decimation-in-frequency (natural-order
// values in, bit-reversed coefficients out), so the zero-padded input of the forward
// decimation-in-time transform is written contiguously and its output is in natural
// order; neither needs a separate bit-reversal pass. Each transform is one pass over
// contiguous 2^11-element blocks plus passes of up to 11 stages over strided groups,
// two stages per shared-memory round trip; results leave the CRT domain in the
// finishing kernels.
#include <algorithm>
#include <vector>

#include "ntt.cuh"

namespace zs {

namespace {
constexpr unsigned kSmemLog = 11;  // 2^11 elements (16 B each) = 32 KB of shared memory per block
constexpr unsigned kThreads = 256;

__device__ __forceinline__ qm31 ldq(const qm31* p) {
  const uint4 r = *reinterpret_cast<const uint4*>(p);
  return qmake(r.x, r.y, r.z, r.w);
}
__device__ __forceinline__ void stq(qm31* p, const qm31& v) {
  *reinterpret_cast<uint4*>(p) = make_uint4(v.a.a, v.a.b, v.b.a, v.b.b);
}
__device__ __forceinline__ cm31 cshl(cm31 x, unsigned k) { return {mshl(x.a, k), mshl(x.b, k)}; }
// The CRT image (u, v) of a QM31 value, held in the a (u) and b (v) slots of a qm31.
ZS_HD qm31 to_crt(const qm31& x) {
  // b s = 2^15 (1 - i)(c + d i) = 2^15 ((c + d) + (d - c) i)
  const cm31 bs = {mshl(madd(x.b.a, x.b.b), 15), mshl(msub(x.b.b, x.b.a), 15)};
  return {cadd(x.a, bs), csub(x.a, bs)};
}
__device__ __forceinline__ qm31 from_crt(const qm31& y) {
  const cm31 a = cshl(cadd(y.a, y.b), 30);  // 2^30 = 1/2
  const cm31 d = csub(y.a, y.b);
  const cm31 b = {mshl(msub(d.a, d.b), 14), mshl(madd(d.a, d.b), 14)};  // (1 + i) d 2^-17
  return {a, b};
}
// Componentwise product in the CRT domain.
__device__ __forceinline__ qm31 crt_mul(const qm31& x, const qm31& y) { return {cmul(x.a, y.a), cmul(x.b, y.b)}; }
__device__ __forceinline__ qm31 crt_add(const qm31& x, const qm31& y) { return {cadd(x.a, y.a), cadd(x.b, y.b)}; }
__device__ __forceinline__ qm31 crt_sub(const qm31& x, const qm31& y) { return {csub(x.a, y.a), csub(x.b, y.b)}; }
__device__ __forceinline__ qm31 crt_neg(const qm31& x) { return {{mneg(x.a.a), mneg(x.a.b)}, {mneg(x.b.a), mneg(x.b.b)}}; }
// Products with the 4th root of unity. w_N^(N/4) = w_4 for every N (the roots are
// powers of one 2-adic root), and its CRT image is J = (i, -i), so J^-1 = (-i, i);
// NttTables checks both. (a + b i) i = -b + a i.
__device__ __forceinline__ qm31 crt_mul_j(const qm31& x) { return {{mneg(x.a.b), x.a.a}, {x.b.b, mneg(x.b.a)}}; }
__device__ __forceinline__ qm31 crt_mul_jinv(const qm31& x) { return {{x.a.b, mneg(x.a.a)}, {mneg(x.b.b), x.b.a}}; }
}  // namespace

// pows[k] = x^k: each thread raises x to its first index, then multiplies along a
// run of kPowRun consecutive powers.
constexpr uint32_t kPowRun = 16;
__global__ void k_qpowers(qm31 x, qm31* pows, uint32_t count) {
  const uint32_t k0 = (blockIdx.x * blockDim.x + threadIdx.x) * kPowRun;
  if (k0 >= count) return;
  qm31 v = qpow(x, k0);
  for (uint32_t k = k0; k < count && k < k0 + kPowRun; ++k) {
    stq(pows + k, v);
    v = qmul(v, x);
  }
}

void qm31_powers(qm31 x, qm31* pows, uint32_t count, cudaStream_t st) {
  if (count == 0) return;
  const uint32_t threads = (count + kPowRun - 1) / kPowRun;
  k_qpowers<<<(threads + kThreads - 1) / kThreads, kThreads, 0, st>>>(x, pows, count);
  ZS_CUDA(cudaGetLastError());
}

__global__ void k_to_crt(const qm31* in, qm31* out, uint32_t count) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < count) stq(out + k, to_crt(ldq(in + k)));
}

NttTables::NttTables(unsigned l, cudaStream_t s) : log_n(l), st(s) {
  if (log_n > 30) throw Error(ZS_EMALFORMED, "NTT size above 2^30");
  {  // the radix-4 passes multiply by J = phi(w_4) = (i, -i) as a rotation of the components
    const qm31 j = to_crt(q_root_of_unity(2)), ji = to_crt(qinv(q_root_of_unity(2)));
    if (!(j.a.a == 0 && j.a.b == 1 && j.b.a == 0 && j.b.b == P - 1 && ji.a.a == 0 && ji.a.b == P - 1 &&
          ji.b.a == 0 && ji.b.b == 1))
      throw Error(ZS_EGENERIC, "unexpected CRT image of the 4th root of unity");
  }
  const uint32_t half = log_n == 0 ? 1 : (1u << (log_n - 1));
  ZS_CUDA(cudaMallocAsync(&fwd, half * sizeof(qm31), st));
  ZS_CUDA(cudaMallocAsync(&inv_crt, half * sizeof(qm31), st));
  ZS_CUDA(cudaMallocAsync(&fwd_crt, half * sizeof(qm31), st));
  const qm31 w = q_root_of_unity(log_n);
  qm31_powers(w, fwd, half, st);
  k_to_crt<<<(half + kThreads - 1) / kThreads, kThreads, 0, st>>>(fwd, fwd_crt, half);
  qm31_powers(qinv(w), inv_crt, half, st);
  k_to_crt<<<(half + kThreads - 1) / kThreads, kThreads, 0, st>>>(inv_crt, inv_crt, half);
  ZS_CUDA(cudaGetLastError());
}
NttTables::~NttTables() {
  cudaFreeAsync(fwd, st);
  cudaFreeAsync(fwd_crt, st);
  cudaFreeAsync(inv_crt, st);
}

// Two stages (b, b + 1) on the four elements m0 + {0, 1, 2, 3} * 2^b of each group in
// shared memory (see k_ntt_pass), one quadruple per thread iteration, then a barrier.
// As a radix-4 step: with t1 = tw[2 i], t2 = tw[i] (i = k 2^(logN - st - 1)) the upper
// pair's twiddle of stage b + 1 is tw[i + N/4] = t2 J (J^-1 in the inverse table), so
// the two stages need three products, by t1, t2 and t3 = t1 t2 = tw[3 i]
// (= -tw[3 i - N/2] past the table's end, w^(N/2) = -1), and one rotation by J:
//   DIT: P = t1 e1, A = t2 e2, B = t3 e3:
//        e0 + P + (A + B), e0 - P + J (A - B), e0 + P - (A + B), e0 - P - J (A - B)
//   DIF: S0 = e0 + e2, S1 = e1 + e3, A = e0 - e2, C = J^-1 (e1 - e3):
//        S0 + S1, t1 (S0 - S1), t2 (A + C), t3 (A - C)
// the same values as the two radix-2 stages, by distributivity.
template <bool DIF>
__device__ __forceinline__ void ntt_radix4(qm31* s, qm31* s_tw, unsigned M, uint32_t G, unsigned lo, unsigned logN,
                                           uint32_t l0, unsigned b, const qm31* __restrict__ tw) {
  const uint32_t hb = 1u << b, total = G << M;
  const unsigned st = lo + 1 + b;
  const size_t half = (size_t)1 << (logN - 1);
  // The stage pair's twiddle triples, (t1, t2, t3) for the G x 2^b distinct k, staged in
  // shared memory first: the global loads are scattered (k << (logN - st - 1)), so all
  // threads issue theirs at once instead of one dependent load per butterfly.
  for (uint32_t e = threadIdx.x; e < (G << b); e += blockDim.x) {
    const uint32_t k = ((e & (hb - 1)) << lo) | (l0 + (e >> b));
    const size_t i2 = (size_t)k << (logN - st - 1), i3 = 3 * i2;
    s_tw[3 * e] = ldq(tw + 2 * i2);
    s_tw[3 * e + 1] = ldq(tw + i2);
    s_tw[3 * e + 2] = i3 < half ? ldq(tw + i3) : crt_neg(ldq(tw + (i3 - half)));
  }
  __syncthreads();
  for (uint32_t q = threadIdx.x; q < (total >> 2); q += blockDim.x) {
    const uint32_t t = q >> (M - 2), r = q & ((1u << (M - 2)) - 1);
    const uint32_t m0 = ((r >> b) << (b + 2)) | (r & (hb - 1));
    const uint32_t e = (t << b) | (r & (hb - 1));
    const qm31 t1 = s_tw[3 * e], t2 = s_tw[3 * e + 1], t3 = s_tw[3 * e + 2];
    qm31* p = s + (t << M) + m0;
    const qm31 e0 = p[0], e1 = p[hb], e2 = p[2 * hb], e3 = p[3 * hb];
    if (!DIF) {
      const qm31 P1 = crt_mul(t1, e1), A = crt_mul(t2, e2), B = crt_mul(t3, e3);
      const qm31 s0 = crt_add(e0, P1), d0 = crt_sub(e0, P1);
      const qm31 sab = crt_add(A, B), jd = crt_mul_j(crt_sub(A, B));
      p[0] = crt_add(s0, sab);
      p[hb] = crt_add(d0, jd);
      p[2 * hb] = crt_sub(s0, sab);
      p[3 * hb] = crt_sub(d0, jd);
    } else {
      const qm31 s0 = crt_add(e0, e2), s1 = crt_add(e1, e3);
      const qm31 a = crt_sub(e0, e2), c = crt_mul_jinv(crt_sub(e1, e3));
      p[0] = crt_add(s0, s1);
      p[hb] = crt_mul(crt_sub(s0, s1), t1);
      p[2 * hb] = crt_mul(crt_add(a, c), t2);
      p[3 * hb] = crt_mul(crt_sub(a, c), t3);
    }
  }
  __syncthreads();
}

// One stage b on the pairs m0 + {0, 1} * 2^b, then a barrier.
template <bool DIF>
__device__ __forceinline__ void ntt_radix2(qm31* s, unsigned M, uint32_t G, unsigned lo, unsigned logN, uint32_t l0,
                                           unsigned b, const qm31* __restrict__ tw) {
  const uint32_t hb = 1u << b, total = G << M;
  const unsigned st = lo + 1 + b;
  for (uint32_t q = threadIdx.x; q < (total >> 1); q += blockDim.x) {
    const uint32_t t = q >> (M - 1), r = q & ((1u << (M - 1)) - 1);
    const uint32_t m0 = ((r >> b) << (b + 1)) | (r & (hb - 1));
    const uint32_t k = ((m0 & (hb - 1)) << lo) | (l0 + t);
    const qm31 tv = ldq(tw + ((size_t)k << (logN - st)));
    qm31* p = s + (t << M) + m0;
    const qm31 x = p[0], y = p[hb];
    if (!DIF) {
      const qm31 u = crt_mul(tv, y);
      p[0] = crt_add(x, u);
      p[hb] = crt_sub(x, u);
    } else {
      p[0] = crt_add(x, y);
      p[hb] = crt_mul(crt_sub(x, y), tv);
    }
  }
  __syncthreads();
}

// out[j] = phi(in[bitrev(j)]) for j < 2^log_n.
__global__ void k_to_crt_brev(const qm31* __restrict__ in, qm31* __restrict__ out, unsigned log_n) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < (1u << log_n)) stq(out + j, to_crt(ldq(in + bitrev(j, log_n))));
}

// x[i] = phi(x[i]) for the elements of C columns (count each), out of place allowed.
__global__ void k_to_crt_cols(const qm31* in, size_t in_stride, qm31* out, size_t out_stride, uint32_t count) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < count)
    stq(out + (size_t)blockIdx.y * out_stride + k, to_crt(ldq(in + (size_t)blockIdx.y * in_stride + k)));
}

// One pass of radix-2/4 butterflies over groups held in shared memory. Global index
// j = (hi << (lo + M)) | (mid << lo) | l with mid < 2^M: a CTA holds the 2^M elements of
// G consecutive l values (one hi), s[t * 2^M + mid], so global stage lo + 1 + b pairs
// mid values that differ in bit b. lo = 0 with G = 1 is a contiguous 2^M block.
// The twiddle of the lower element j at stage st is tw[(j mod 2^(st-1)) << (logN - st)]
// in both directions:
//   DIT (bit-reversed in, natural out), stages ascending:  x, y -> x + t y, x - t y;
//   DIF (natural in, bit-reversed out), stages descending: x, y -> x + y, (x - y) t.
// Local stages [b_lo, b_hi) run two at a time (four elements per thread in registers)
// with a barrier per pair. Where the pass reads its input (`in_mode`): kInPlace `a`;
// kToCrt QM31 values of `src` mapped into the CRT domain; kExpand `src[j >> expand]`, the
// compact values whose 2^expand copies the first `expand` stages of a zero-padded DIT
// would make. `to_qm31`: the pass leaves the CRT domain on its store (the last pass).
enum InMode : unsigned { kInPlace = 0, kToCrt = 1, kExpand = 2 };
template <bool DIF>
__global__ void __launch_bounds__(kThreads) k_ntt_pass(qm31* a, size_t stride, const qm31* __restrict__ src,
                                                       size_t src_stride, unsigned in_mode, unsigned expand,
                                                       unsigned to_qm31, unsigned logN, unsigned lo, unsigned M,
                                                       unsigned G, unsigned b_lo, unsigned b_hi,
                                                       const qm31* __restrict__ tw) {
  extern __shared__ uint4 smem_raw[];
  qm31* s = reinterpret_cast<qm31*>(smem_raw);
  qm31* s_tw = s + ((size_t)G << M);
  const uint32_t gpl = (1u << lo) / G;  // CTAs per hi value
  const uint32_t hi = blockIdx.x / gpl, l0 = (blockIdx.x % gpl) * G;
  const size_t off = ((size_t)hi << (lo + M)) + l0;
  qm31* col = a + (size_t)blockIdx.y * stride + off;
  const uint32_t total = G << M;
  const unsigned lg_g = 31 - __clz(G);
  if (in_mode == kToCrt) {
    const qm31* in = src + (size_t)blockIdx.y * src_stride + off;
    for (uint32_t idx = threadIdx.x; idx < total; idx += blockDim.x) {
      const uint32_t t = idx & (G - 1), mid = idx >> lg_g;
      s[(t << M) + mid] = to_crt(ldq(in + ((size_t)mid << lo) + t));
    }
  } else if (in_mode == kExpand) {
    const qm31* in = src + (size_t)blockIdx.y * src_stride;
    for (uint32_t idx = threadIdx.x; idx < total; idx += blockDim.x) {
      const uint32_t t = idx & (G - 1), mid = idx >> lg_g;
      s[(t << M) + mid] = ldq(in + ((off + ((size_t)mid << lo) + t) >> expand));
    }
  } else {
    for (uint32_t idx = threadIdx.x; idx < total; idx += blockDim.x) {
      const uint32_t t = idx & (G - 1), mid = idx >> lg_g;
      s[(t << M) + mid] = ldq(col + ((size_t)mid << lo) + t);
    }
  }
  __syncthreads();
  if (!DIF) {
    unsigned b = b_lo;
    for (; b + 1 < b_hi; b += 2) ntt_radix4<false>(s, s_tw, M, G, lo, logN, l0, b, tw);
    if (b < b_hi) ntt_radix2<false>(s, M, G, lo, logN, l0, b, tw);
  } else {
    int b = (int)b_hi - 1;
    for (; b - 1 >= (int)b_lo; b -= 2) ntt_radix4<true>(s, s_tw, M, G, lo, logN, l0, (unsigned)(b - 1), tw);
    if (b >= (int)b_lo) ntt_radix2<true>(s, M, G, lo, logN, l0, (unsigned)b, tw);
  }
  for (uint32_t idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const uint32_t t = idx & (G - 1), mid = idx >> lg_g;
    const qm31 v = s[(t << M) + mid];
    stq(col + ((size_t)mid << lo) + t, to_qm31 ? from_crt(v) : v);
  }
}

// The passes of a size-2^logN transform: one over contiguous 2^S-element blocks
// (S = min(logN, 11), stages 1..S) and passes of up to 11 stages over strided groups
// (2048 elements, 32 KB, per CTA, or two groups of 2^11 at M = 11) for stages
// S+1..logN; smaller CTAs keep more of them resident to cover the twiddle loads.
struct PassPlan {
  unsigned lo, M;
  uint32_t G;
};
static std::vector<PassPlan> plan_passes(unsigned logN) {
  std::vector<PassPlan> v;
  const unsigned S = logN < kSmemLog ? logN : kSmemLog;
  v.push_back({0, S, 1});
  unsigned lo = S;
  while (lo < logN) {
    const unsigned rem = logN - lo, passes = (rem + kSmemLog - 1) / kSmemLog;
    const unsigned M = (rem + passes - 1) / passes;
    uint32_t G = 2048u >> M;
    if (G < 2) G = 2;
    if (G > (1u << lo)) G = 1u << lo;
    v.push_back({lo, M, G});
    lo += M;
  }
  return v;
}

// Shared memory of a pass: its 2^M x G elements and the twiddle triples of its widest
// stage pair (G x 2^(M-2) of them).
static size_t pass_smem(const PassPlan& p) {
  return (((size_t)p.G << p.M) + (p.M >= 2 ? (size_t)3 * (p.G << (p.M - 2)) : 0)) * sizeof(qm31);
}

template <bool DIF>
static void launch_pass(qm31* a, size_t stride, const qm31* src, size_t src_stride, unsigned in_mode,
                        unsigned expand, bool to_qm31, uint32_t C, unsigned logN, const PassPlan& p, unsigned b_lo,
                        unsigned b_hi, const qm31* tw, cudaStream_t st) {
  static const bool attr = [] {  // 64 KB of elements + 48 KB of twiddles at most (M = 11, G = 2)
    ZS_CUDA(cudaFuncSetAttribute(k_ntt_pass<DIF>, cudaFuncAttributeMaxDynamicSharedMemorySize, 114688));
    return true;
  }();
  (void)attr;
  const uint32_t ctas = (1u << (logN - p.M)) / p.G;
  k_ntt_pass<DIF><<<dim3(ctas, C), kThreads, pass_smem(p), st>>>(a, stride, src, src_stride, in_mode, expand,
                                                                 to_qm31 ? 1u : 0u, logN, p.lo, p.M, p.G, b_lo, b_hi,
                                                                 tw);
}

// Forward DIT stages first..logN (natural output, QM31 values: the last pass leaves the
// CRT domain). The first `first - 1` stages of the zero-padded input only copy: the
// first pass reads the compact CRT-domain values `src` (value j at 2^(first-1) positions).
static void dit_stages(qm31* a, size_t stride, const qm31* src, size_t src_stride, uint32_t C, unsigned logN,
                       const qm31* tw, cudaStream_t st, unsigned first) {
  if (logN == 0) throw Error(ZS_EGENERIC, "dit_stages: empty transform");
  const std::vector<PassPlan> plan = plan_passes(logN);
  bool first_pass = true;
  for (size_t i = 0; i < plan.size(); ++i) {
    const PassPlan& p = plan[i];
    const unsigned s_lo = p.lo + 1, s_hi = p.lo + p.M;  // global stages of this pass
    if (s_hi < first && i + 1 < plan.size()) continue;
    // (first > logN: every stage copies; the last pass only expands and leaves the CRT domain)
    const unsigned b_lo = first > s_lo ? std::min(first - s_lo, p.M) : 0;
    launch_pass<false>(a, stride, first_pass ? src : nullptr, src_stride, first_pass ? kExpand : kInPlace,
                       first - 1, i + 1 == plan.size(), C, logN, p, b_lo, p.M, tw, st);
    first_pass = false;
  }
  ZS_CUDA(cudaGetLastError());
}

// Inverse DIF over all stages: natural-order QM31 values in `src` (mapped into the CRT
// domain by the first pass), bit-reversed CRT-domain output in `a`.
static void dif_all(const qm31* src, size_t src_stride, qm31* a, size_t stride, uint32_t C, unsigned logN,
                    const qm31* tw, cudaStream_t st) {
  if (logN == 0) {
    k_to_crt_cols<<<dim3(1, C), 32, 0, st>>>(src, src_stride, a, stride, 1);
    ZS_CUDA(cudaGetLastError());
    return;
  }
  const std::vector<PassPlan> plan = plan_passes(logN);
  for (size_t i = plan.size(); i-- > 0;) {
    const bool first = i + 1 == plan.size();
    launch_pass<true>(a, stride, first ? src : nullptr, src_stride, first ? kToCrt : kInPlace, 0, false, C, logN,
                      plan[i], 0, plan[i].M, tw, st);
  }
  ZS_CUDA(cudaGetLastError());
}

// The inverse DIF leaves phi(n c_k) at position j = bitrev_n(k). For each j:
// coeffs[c][j] = c_k (QM31, kept in bit-reversed order), and the forward input
// phi(c_k offset^k) belongs at position bitrev_N(k) = j << B of the size-N transform. That
// input is zero elsewhere, so its first B stages only copy the value across the 2^B block
// at j << B: the value goes to wbuf[c][j] once, and the forward transform's first pass
// reads it for all 2^B positions and starts at stage B + 1.
// offset_crt[j] = phi(offset^bitrev_n(j)) (bit-reversed, so every read is coalesced).
__global__ void k_coeff_finish(qm31* coeffs, size_t c_stride, qm31* wbuf, size_t w_stride, unsigned log_n,
                               const qm31* __restrict__ offset_crt) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= (1u << log_n)) return;
  qm31* cp = coeffs + (size_t)blockIdx.y * c_stride + j;
  qm31 v = ldq(cp);
  const unsigned sh = (31 - log_n) % 31;
  v = qmake(mshl(v.a.a, sh), mshl(v.a.b, sh), mshl(v.b.a, sh), mshl(v.b.b, sh));
  stq(cp, from_crt(v));
  stq(wbuf + (size_t)blockIdx.y * w_stride + j, crt_mul(v, ldq(offset_crt + j)));
}

void lde_qm31(const qm31* values, size_t v_stride, qm31* coeffs, size_t c_stride, qm31* codeword, size_t w_stride,
              uint32_t C, const NttTables& small, const NttTables& big, const qm31* offset_pows, cudaStream_t st) {
  const unsigned log_n = small.log_n, log_N = big.log_n;
  const uint32_t n = 1u << log_n;
  if (log_N == 0) throw Error(ZS_EMALFORMED, "LDE onto a domain of one point");
  // inverse transform on H: natural-order values in, bit-reversed CRT-domain n c_k out
  dif_all(values, v_stride, coeffs, c_stride, C, log_n, small.inv_crt, st);
  // scale by 1/n, leave the CRT domain for the coefficients, and keep the forward
  // input compact for the forward transform's first pass
  qm31 *off_crt = nullptr, *wbuf = nullptr;
  ZS_CUDA(cudaMallocAsync((void**)&off_crt, (size_t)n * sizeof(qm31), st));
  ZS_CUDA(cudaMallocAsync((void**)&wbuf, (size_t)C * n * sizeof(qm31), st));
  k_to_crt_brev<<<(n + kThreads - 1) / kThreads, kThreads, 0, st>>>(offset_pows, off_crt, log_n);
  k_coeff_finish<<<dim3((n + kThreads - 1) / kThreads, C), kThreads, 0, st>>>(coeffs, c_stride, wbuf, n, log_n,
                                                                              off_crt);
  ZS_CUDA(cudaGetLastError());
  dit_stages(codeword, w_stride, wbuf, n, C, log_N, big.fwd_crt, st, log_N - log_n + 1);
  ZS_CUDA(cudaFreeAsync(wbuf, st));
  ZS_CUDA(cudaFreeAsync(off_crt, st));
}

}  // namespace zs
