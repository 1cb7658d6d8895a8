// Radix-2 NTT over QM31 on the device: the prover's interpolation on H and
// evaluation on D (src/m31/poly/univariate.zig:11-19, 79-139 compute the same unique
// polynomial and the same evaluations, O(n^2) / O(n N) on the CPU).
#pragma once
#include "common.cuh"

namespace zs {

// Powers of a primitive 2^log_n-th root w (qm31.zig:86-89): fwd[k] = w^k and
// inv[k] = w^-k for k < 2^(log_n-1).
struct NttTables {
  unsigned log_n = 0;
  qm31* fwd = nullptr;      // w^k, k < n/2 (QM31; the domain points of D)
  qm31* fwd_crt = nullptr;  // phi(w^k): forward twiddles in the CRT domain (ntt.cu)
  qm31* inv_crt = nullptr;  // phi(w^-k)
  cudaStream_t st = nullptr;  // freed in stream order, so concurrent provers never synchronize the device
  NttTables(unsigned log_n, cudaStream_t st);
  ~NttTables();
  NttTables(const NttTables&) = delete;
  NttTables& operator=(const NttTables&) = delete;
};

// Low-degree extension of C columns of 2^log_n trace values (natural order on
// H = <w_n>) to 2^log_N evaluations on D = offset * <w_N> (natural order), keeping the
// coefficients in bit-reversed order: coeffs[c][j] = coefficient bitrev(j) of the
// interpolation of values[c] on H; codeword[c][i] = f_c(d_i).
// offset_pows: offset^k for k < 2^log_n.
void lde_qm31(const qm31* values, size_t v_stride, qm31* coeffs, size_t c_stride, qm31* codeword, size_t w_stride,
              uint32_t C, const NttTables& small, const NttTables& big, const qm31* offset_pows, cudaStream_t st);

// pows[k] = x^k for k < count.
void qm31_powers(qm31 x, qm31* pows, uint32_t count, cudaStream_t st);

}  // namespace zs
