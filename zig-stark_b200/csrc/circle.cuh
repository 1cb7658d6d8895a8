// Circle FFT over M31 on the device (see circle.cu).
#pragma once
#include "common.cuh"

namespace zs {

// Twiddle tables of the canonic circle domain of size 2^lg (coset.zig:59-65
// canonicHalf(lg) plus its conjugate), forward and inverse, resident on the device.
struct CircleDomain {
  unsigned lg;
  uint32_t* tw = nullptr;   // flat forward table, n words, each twiddle doubled (circle.cu)
  uint32_t* itw = nullptr;  // elementwise inverses, doubled
  // The canonic domain canonicHalf(lg) ++ conjugate.
  CircleDomain(unsigned lg, cudaStream_t st);
  // The domain half_coset ++ conjugate of the half coset {offset + k * step, k < 2^(lg-1)}.
  CircleDomain(unsigned lg, cpoint offset, cpoint step, cudaStream_t st);
  ~CircleDomain();
  CircleDomain(const CircleDomain&) = delete;
  CircleDomain& operator=(const CircleDomain&) = delete;

 private:
  void init(cpoint offset, cpoint step, cudaStream_t st);
};

void canonic_half(unsigned lg, cpoint* offset, cpoint* step);

// Words of scratch circle_lde needs for C columns.
size_t lde_scratch_words(unsigned L, unsigned B, uint32_t C);

// Low-degree extension of C columns of 2^L natural-order evaluations on the
// canonic domain of size 2^L to natural-order evaluations on the canonic domain of
// size 2^(L+B): circleIFFT, zero-pad A and B separately, circleFFT
// (src/m31/ntt/circle.zig:195-346). Column c of the input starts at
// d_in + c * in_stride, of the output at d_out + c * out_stride.
void circle_lde(const uint32_t* d_in, size_t in_stride, uint32_t* d_out, size_t out_stride, uint32_t C, unsigned L,
                unsigned B, const CircleDomain& small, const CircleDomain& big, uint32_t* scratch, cudaStream_t st);

// circleFFT / circleIFFT of C contiguous columns of 2^dom.lg words (coefficients in
// the reference's A-then-B layout). scratch: C * 2^lg words.
void circle_fft(const uint32_t* d_coeffs, uint32_t* d_evals, uint32_t C, const CircleDomain& dom, uint32_t* scratch,
                cudaStream_t st);
void circle_ifft(const uint32_t* d_evals, uint32_t* d_coeffs, uint32_t C, const CircleDomain& dom, uint32_t* scratch,
                 cudaStream_t st);

// Forward and inverse tables of the canonic domain of size 2^lg written into caller
// memory (2^lg words each), and circle_lde with the tables passed directly
// (itw_small: inverse table of the 2^L domain, tw_big: forward table of the 2^(L+B)
// domain; scratch: lde_scratch_words(L, B, C) words).
void circle_twiddles_into(unsigned lg, uint32_t* tw, uint32_t* itw, cudaStream_t st);
void circle_lde_tables(const uint32_t* d_in, size_t in_stride, uint32_t* d_out, size_t out_stride, uint32_t C,
                       unsigned L, unsigned B, const uint32_t* itw_small, const uint32_t* tw_big, uint32_t* scratch,
                       cudaStream_t st);

}  // namespace zs
