// Radix-2 decimation-in-time NTT over QM31. QM31 is the ring CM31[j]/(j^2+i); both
// of its CM31 components see the 2-adic root with order 2^32, so the DFT over a
// 2-power subgroup is invertible and equals the reference's Lagrange interpolation /
// Horner evaluation value for value.
//
// A transform of 2^logN points: a bit-reversed load, stages 2..2^S inside 2^S-point
// blocks held in shared memory (S <= 11), then one global pass per larger stage.
#include "ntt.cuh"

namespace zs {

namespace {
constexpr unsigned kSmemLog = 11;  // 2^11 QM31 = 32 KB of shared memory per block
constexpr unsigned kThreads = 256;

__device__ __forceinline__ qm31 ldq(const qm31* p) {
  const uint4 r = *reinterpret_cast<const uint4*>(p);
  return qmake(r.x, r.y, r.z, r.w);
}
__device__ __forceinline__ void stq(qm31* p, const qm31& v) {
  *reinterpret_cast<uint4*>(p) = make_uint4(v.a.a, v.a.b, v.b.a, v.b.b);
}
}  // namespace

__global__ void k_qpowers(qm31 x, qm31* pows, uint32_t count) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < count) stq(pows + k, qpow(x, k));
}

void qm31_powers(qm31 x, qm31* pows, uint32_t count, cudaStream_t st) {
  if (count == 0) return;
  k_qpowers<<<(count + kThreads - 1) / kThreads, kThreads, 0, st>>>(x, pows, count);
  ZS_CUDA(cudaGetLastError());
}

NttTables::NttTables(unsigned l, cudaStream_t s) : log_n(l), st(s) {
  if (log_n > 30) throw Error(ZS_EMALFORMED, "NTT size above 2^30");
  const uint32_t half = log_n == 0 ? 1 : (1u << (log_n - 1));
  ZS_CUDA(cudaMallocAsync(&fwd, half * sizeof(qm31), st));
  ZS_CUDA(cudaMallocAsync(&inv, half * sizeof(qm31), st));
  const qm31 w = q_root_of_unity(log_n);
  qm31_powers(w, fwd, half, st);
  qm31_powers(qinv(w), inv, half, st);
}
NttTables::~NttTables() {
  cudaFreeAsync(fwd, st);
  cudaFreeAsync(inv, st);
}

// dst[bitrev(i)] = src[i], i < 2^logN.
__global__ void k_bitrev_load(const qm31* __restrict__ src, size_t s_stride, qm31* __restrict__ dst, size_t d_stride,
                              unsigned logN) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (1u << logN)) return;
  const qm31* s = src + (size_t)blockIdx.y * s_stride;
  qm31* d = dst + (size_t)blockIdx.y * d_stride;
  stq(d + bitrev(i, logN), ldq(s + i));
}

// Stages 1..S (len 2..2^S) inside 2^S-point blocks.
__global__ void __launch_bounds__(kThreads) k_ntt_smem(qm31* a, size_t stride, unsigned logN, unsigned S,
                                                       const qm31* __restrict__ tw) {
  extern __shared__ uint4 smem_raw[];
  qm31* s = reinterpret_cast<qm31*>(smem_raw);
  const uint32_t B = 1u << S;
  qm31* col = a + (size_t)blockIdx.y * stride + (size_t)blockIdx.x * B;
  for (uint32_t i = threadIdx.x; i < B; i += blockDim.x) s[i] = ldq(col + i);
  __syncthreads();
  for (unsigned st = 1; st <= S; ++st) {
    const uint32_t half = 1u << (st - 1);
    for (uint32_t b = threadIdx.x; b < (B >> 1); b += blockDim.x) {
      const uint32_t k = b & (half - 1);
      const uint32_t j = ((b >> (st - 1)) << st) + k;
      const qm31 t = qmul(ldq(tw + ((size_t)k << (logN - st))), s[j + half]);
      const qm31 u = s[j];
      s[j] = qadd(u, t);
      s[j + half] = qsub(u, t);
    }
    __syncthreads();
  }
  for (uint32_t i = threadIdx.x; i < B; i += blockDim.x) stq(col + i, s[i]);
}

// One global stage of length 2^st.
__global__ void k_ntt_stage(qm31* a, size_t stride, unsigned logN, unsigned st, const qm31* __restrict__ tw) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= (1u << (logN - 1))) return;
  qm31* col = a + (size_t)blockIdx.y * stride;
  const uint32_t half = 1u << (st - 1);
  const uint32_t k = b & (half - 1);
  const uint32_t j = ((b >> (st - 1)) << st) + k;
  const qm31 t = qmul(ldq(tw + ((size_t)k << (logN - st))), ldq(col + j + half));
  const qm31 u = ldq(col + j);
  stq(col + j, qadd(u, t));
  stq(col + j + half, qsub(u, t));
}

// x[i] *= 2^shift (an M31 scalar, used for 1/n = 2^(31 - log n)).
__global__ void k_scale(qm31* a, size_t stride, uint32_t n, unsigned shift) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  qm31* p = a + (size_t)blockIdx.y * stride + i;
  qm31 v = ldq(p);
  v = qmake(mshl(v.a.a, shift), mshl(v.a.b, shift), mshl(v.b.a, shift), mshl(v.b.b, shift));
  stq(p, v);
}

static void run_stages(qm31* a, size_t stride, uint32_t C, unsigned logN, const qm31* tw, cudaStream_t st) {
  if (logN == 0) return;
  const unsigned S = logN < kSmemLog ? logN : kSmemLog;
  const uint32_t B = 1u << S;
  k_ntt_smem<<<dim3((1u << logN) / B, C), kThreads, B * sizeof(qm31), st>>>(a, stride, logN, S, tw);
  for (unsigned s = S + 1; s <= logN; ++s) {
    const uint32_t half = 1u << (logN - 1);
    k_ntt_stage<<<dim3((half + kThreads - 1) / kThreads, C), kThreads, 0, st>>>(a, stride, logN, s, tw);
  }
}

void ntt(const qm31* in, qm31* out, size_t stride, uint32_t C, const NttTables& t, bool inverse, cudaStream_t st) {
  const unsigned logN = t.log_n;
  const uint32_t N = 1u << logN;
  if (in == out) throw Error(ZS_EGENERIC, "ntt: in-place transform needs a separate buffer for the bit reversal");
  k_bitrev_load<<<dim3((N + kThreads - 1) / kThreads, C), kThreads, 0, st>>>(in, stride, out, stride, logN);
  run_stages(out, stride, C, logN, inverse ? t.inv : t.fwd, st);
  if (inverse && logN > 0)
    k_scale<<<dim3((N + kThreads - 1) / kThreads, C), kThreads, 0, st>>>(out, stride, N, (31 - logN) % 31);
  ZS_CUDA(cudaGetLastError());
}

// coeffs[c][k] = scaled inverse-transform result (in place); big[c][bitrev_N(k)] =
// coeffs[c][k] * offset^k for k < n (the rest of `big` was zeroed).
__global__ void k_coeff_finish(qm31* coeffs, size_t c_stride, qm31* big, size_t b_stride, unsigned log_n,
                               unsigned log_N, const qm31* __restrict__ offset_pows) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (1u << log_n)) return;
  qm31* cp = coeffs + (size_t)blockIdx.y * c_stride + k;
  qm31 v = ldq(cp);
  const unsigned sh = (31 - log_n) % 31;
  v = qmake(mshl(v.a.a, sh), mshl(v.a.b, sh), mshl(v.b.a, sh), mshl(v.b.b, sh));
  stq(cp, v);
  stq(big + (size_t)blockIdx.y * b_stride + bitrev(k, log_N), qmul(v, ldq(offset_pows + k)));
}

void lde_qm31(const qm31* values, size_t v_stride, qm31* coeffs, size_t c_stride, qm31* codeword, size_t w_stride,
              uint32_t C, const NttTables& small, const NttTables& big, const qm31* offset_pows, cudaStream_t st) {
  const unsigned log_n = small.log_n, log_N = big.log_n;
  const uint32_t n = 1u << log_n;
  // inverse transform on H (bit-reversed load, stages, scaling folded into the finish)
  k_bitrev_load<<<dim3((n + kThreads - 1) / kThreads, C), kThreads, 0, st>>>(values, v_stride, coeffs, c_stride,
                                                                             log_n);
  run_stages(coeffs, c_stride, C, log_n, small.inv, st);
  for (uint32_t c = 0; c < C; ++c)
    ZS_CUDA(cudaMemsetAsync(codeword + (size_t)c * w_stride, 0, ((size_t)1 << log_N) * sizeof(qm31), st));
  k_coeff_finish<<<dim3((n + kThreads - 1) / kThreads, C), kThreads, 0, st>>>(coeffs, c_stride, codeword, w_stride,
                                                                              log_n, log_N, offset_pows);
  run_stages(codeword, w_stride, C, log_N, big.fwd, st);
  ZS_CUDA(cudaGetLastError());
}

}  // namespace zs
