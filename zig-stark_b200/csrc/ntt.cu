// Radix-2 decimation-in-time NTT over QM31, computed in the CRT domain.
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
// A transform of 2^logN points: a bit-reversed load (with phi), stages 2..2^S inside
// 2^S-point blocks held in shared memory (S <= 11), then one global pass per larger
// stage; results leave the CRT domain in the finishing kernels.
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
__device__ __forceinline__ qm31 to_crt(const qm31& x) {
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

// dst[bitrev(i)] = phi(src[i]), i < 2^logN.
__global__ void k_bitrev_load(const qm31* __restrict__ src, size_t s_stride, qm31* __restrict__ dst, size_t d_stride,
                              unsigned logN) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (1u << logN)) return;
  const qm31* s = src + (size_t)blockIdx.y * s_stride;
  qm31* d = dst + (size_t)blockIdx.y * d_stride;
  stq(d + bitrev(i, logN), to_crt(ldq(s + i)));
}

// Stages first..S (len 2^first..2^S) inside 2^S-point blocks, CRT domain.
__global__ void __launch_bounds__(kThreads) k_ntt_smem(qm31* a, size_t stride, unsigned logN, unsigned first,
                                                       unsigned S, const qm31* __restrict__ tw) {
  extern __shared__ uint4 smem_raw[];
  qm31* s = reinterpret_cast<qm31*>(smem_raw);
  const uint32_t B = 1u << S;
  qm31* col = a + (size_t)blockIdx.y * stride + (size_t)blockIdx.x * B;
  for (uint32_t i = threadIdx.x; i < B; i += blockDim.x) s[i] = ldq(col + i);
  __syncthreads();
  for (unsigned st = first; st <= S; ++st) {
    const uint32_t half = 1u << (st - 1);
    for (uint32_t b = threadIdx.x; b < (B >> 1); b += blockDim.x) {
      const uint32_t k = b & (half - 1);
      const uint32_t j = ((b >> (st - 1)) << st) + k;
      const qm31 t = crt_mul(ldq(tw + ((size_t)k << (logN - st))), s[j + half]);
      const qm31 u = s[j];
      s[j] = crt_add(u, t);
      s[j + half] = crt_sub(u, t);
    }
    __syncthreads();
  }
  for (uint32_t i = threadIdx.x; i < B; i += blockDim.x) stq(col + i, s[i]);
}

// Stages lo+1..lo+M in one pass: index j = (hi << (lo + M)) | (mid << lo) | l with
// mid < 2^M; a CTA holds the 2^M elements of G consecutive l values (one hi) in shared
// memory, so a stage's butterflies pair mid values that differ in one bit. The twiddle
// of the lower element j at stage lo + 1 + b is tw[(j mod 2^(lo + b)) << (logN - lo - 1 - b)].
__global__ void __launch_bounds__(kThreads) k_ntt_strided(qm31* a, size_t stride, unsigned logN, unsigned lo,
                                                          unsigned M, unsigned G, const qm31* __restrict__ tw) {
  extern __shared__ uint4 smem_raw[];
  qm31* s = reinterpret_cast<qm31*>(smem_raw);  // s[t * 2^M + mid]
  const uint32_t lcount = 1u << lo, gpl = lcount / G;  // CTAs per hi value
  const uint32_t hi = blockIdx.x / gpl, l0 = (blockIdx.x % gpl) * G;
  qm31* col = a + (size_t)blockIdx.y * stride + ((size_t)hi << (lo + M)) + l0;
  const uint32_t total = G << M;
  const unsigned lg_g = 31 - __clz(G);
  for (uint32_t idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const uint32_t t = idx & (G - 1), mid = idx >> lg_g;
    s[(t << M) + mid] = ldq(col + ((size_t)mid << lo) + t);
  }
  __syncthreads();
  for (unsigned b = 0; b < M; ++b) {
    const unsigned st = lo + 1 + b;
    const uint32_t half = 1u << b;
    for (uint32_t q = threadIdx.x; q < (total >> 1); q += blockDim.x) {
      const uint32_t t = q >> (M - 1), r = q & ((1u << (M - 1)) - 1);
      const uint32_t m0 = ((r >> b) << (b + 1)) | (r & (half - 1));
      const uint32_t k = ((m0 & (half - 1)) << lo) | (l0 + t);
      qm31* p = s + (t << M) + m0;
      const qm31 tv = crt_mul(ldq(tw + ((size_t)k << (logN - st))), p[half]);
      const qm31 u = p[0];
      p[0] = crt_add(u, tv);
      p[half] = crt_sub(u, tv);
    }
    __syncthreads();
  }
  for (uint32_t idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const uint32_t t = idx & (G - 1), mid = idx >> lg_g;
    stq(col + ((size_t)mid << lo) + t, s[(t << M) + mid]);
  }
}

// x[i] = phi^-1(x[i]) * 2^shift (2^shift an M31 scalar: 1/n = 2^(31 - log n), or 1).
__global__ void k_from_crt(qm31* a, size_t stride, uint32_t n, unsigned shift) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  qm31* p = a + (size_t)blockIdx.y * stride + i;
  qm31 v = from_crt(ldq(p));
  if (shift) v = qmake(mshl(v.a.a, shift), mshl(v.a.b, shift), mshl(v.b.a, shift), mshl(v.b.b, shift));
  stq(p, v);
}

// Stages first..logN of a transform whose stages below `first` are done: one
// shared-memory pass over 2^11-point blocks, then passes of up to 11 stages over
// strided groups (at most 4096 elements, 64 KB, per CTA).
static void run_stages(qm31* a, size_t stride, uint32_t C, unsigned logN, const qm31* tw, cudaStream_t st,
                       unsigned first = 1) {
  if (logN == 0 || first > logN) return;
  const unsigned S = logN < kSmemLog ? logN : kSmemLog;
  if (first <= S) {
    const uint32_t B = 1u << S;
    k_ntt_smem<<<dim3((1u << logN) / B, C), kThreads, B * sizeof(qm31), st>>>(a, stride, logN, first, S, tw);
  }
  unsigned lo = S > first - 1 ? S : first - 1;
  while (lo < logN) {
    const unsigned rem = logN - lo, passes = (rem + kSmemLog - 1) / kSmemLog;
    const unsigned M = (rem + passes - 1) / passes;
    uint32_t G = 4096u >> M;
    if (G < 2) G = 2;
    if (G > (1u << lo)) G = 1u << lo;
    const size_t sb = ((size_t)G << M) * sizeof(qm31);
    const uint32_t ctas = (1u << (logN - M)) / G;
    ZS_CUDA(cudaFuncSetAttribute(k_ntt_strided, cudaFuncAttributeMaxDynamicSharedMemorySize, 65536));
    k_ntt_strided<<<dim3(ctas, C), kThreads, sb, st>>>(a, stride, logN, lo, M, G, tw);
    lo += M;
  }
  ZS_CUDA(cudaGetLastError());
}

void ntt(const qm31* in, qm31* out, size_t stride, uint32_t C, const NttTables& t, bool inverse, cudaStream_t st) {
  const unsigned logN = t.log_n;
  const uint32_t N = 1u << logN;
  if (in == out) throw Error(ZS_EGENERIC, "ntt: in-place transform needs a separate buffer for the bit reversal");
  k_bitrev_load<<<dim3((N + kThreads - 1) / kThreads, C), kThreads, 0, st>>>(in, stride, out, stride, logN);
  run_stages(out, stride, C, logN, inverse ? t.inv_crt : t.fwd_crt, st);
  k_from_crt<<<dim3((N + kThreads - 1) / kThreads, C), kThreads, 0, st>>>(out, stride, N,
                                                                          inverse ? (31 - logN) % 31 : 0);
  ZS_CUDA(cudaGetLastError());
}

// coeffs[c][k] = phi^-1 of the scaled inverse-transform result (in place), and
// v = phi(coeffs[c][k] * offset^k) for k < n goes to the bit-reversed input of the
// size-N forward transform. That input is zero except at position bitrev_N(k) =
// bitrev_n(k) << B, so its first B stages only copy v across the 2^B-element block
// (each stage pairs a filled element with a zero one): the block is written as 2^B
// copies of v and the forward transform starts at stage B + 1. offset_crt[k] = phi(offset^k).
__global__ void k_coeff_finish(qm31* coeffs, size_t c_stride, qm31* big, size_t b_stride, unsigned log_n,
                               unsigned log_N, const qm31* __restrict__ offset_crt) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (1u << log_n)) return;
  qm31* cp = coeffs + (size_t)blockIdx.y * c_stride + k;
  qm31 v = ldq(cp);
  const unsigned sh = (31 - log_n) % 31;
  v = qmake(mshl(v.a.a, sh), mshl(v.a.b, sh), mshl(v.b.a, sh), mshl(v.b.b, sh));
  stq(cp, from_crt(v));
  const qm31 w = crt_mul(v, ldq(offset_crt + k));
  const unsigned B = log_N - log_n;
  qm31* dst = big + (size_t)blockIdx.y * b_stride + ((size_t)bitrev(k, log_n) << B);
  for (uint32_t r = 0; r < (1u << B); ++r) stq(dst + r, w);
}

void lde_qm31(const qm31* values, size_t v_stride, qm31* coeffs, size_t c_stride, qm31* codeword, size_t w_stride,
              uint32_t C, const NttTables& small, const NttTables& big, const qm31* offset_pows, cudaStream_t st) {
  const unsigned log_n = small.log_n, log_N = big.log_n;
  const uint32_t n = 1u << log_n, N = 1u << log_N;
  // inverse transform on H (bit-reversed load into the CRT domain, stages)
  k_bitrev_load<<<dim3((n + kThreads - 1) / kThreads, C), kThreads, 0, st>>>(values, v_stride, coeffs, c_stride,
                                                                             log_n);
  run_stages(coeffs, c_stride, C, log_n, small.inv_crt, st);
  // scale by 1/n, leave the CRT domain for the coefficients, and fill the forward
  // input after its first log_N - log_n stages
  qm31* off_crt = nullptr;
  ZS_CUDA(cudaMallocAsync((void**)&off_crt, (size_t)n * sizeof(qm31), st));
  k_to_crt<<<(n + kThreads - 1) / kThreads, kThreads, 0, st>>>(offset_pows, off_crt, n);
  k_coeff_finish<<<dim3((n + kThreads - 1) / kThreads, C), kThreads, 0, st>>>(coeffs, c_stride, codeword, w_stride,
                                                                              log_n, log_N, off_crt);
  ZS_CUDA(cudaFreeAsync(off_crt, st));
  run_stages(codeword, w_stride, C, log_N, big.fwd_crt, st, log_N - log_n + 1);
  k_from_crt<<<dim3((N + kThreads - 1) / kThreads, C), kThreads, 0, st>>>(codeword, w_stride, N, 0);
  ZS_CUDA(cudaGetLastError());
}

}  // namespace zs
