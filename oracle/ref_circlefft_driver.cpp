// ORACLE — test and benchmark infrastructure only. Host side of the reference's own
// GPU circle FFT, so that its kernels (src/cuda/kernels/circlefft.cu, compiled from
// the reference's source for sm_100a by oracle/build_ref.sh into oracle/_ref/) can be
// checked against the oracle and timed beside this library's transform on the same
// B200.
//
// This restates src/cuda/circlefft_gpu.zig:46-175 call for call: per call it
// allocates the device buffers, builds the twiddle tree on the host with the CPU
// transform's own functions (precomputeTwiddles, lineTwiddleSlice, circleTwiddles:
// src/m31/ntt/circle.zig:65-106, restated in oracle/circle.hpp), copies the input and
// the twiddles to the device, launches one kernel per butterfly layer (256 threads
// per block, src/cuda/circlefft_gpu.zig:41-43), bit-reverses, and copies the result
// back. The reference creates its own context (src/cuda/cuda.zig); this driver uses the
// device's primary context so it can share a process with the CUDA runtime.
//
// Exported (extern "C"):
//   ref_cfft_init(cubin_path)            load the module; 0 on success
//   ref_cfft_fft(coeffs, evals, lg, t)   circleFFT on canonicHalf(lg), t[0] = wall ms of
//                                        the whole call, t[1] = device ms of its launches
//   ref_cfft_ifft(evals, coeffs, lg, t)  circleIFFT, same timings
//   ref_cfft_twiddles(fast)              1 = build the twiddle tree by walking the coset
//                                        (same values; for sizes where the reference's
//                                        per-point evaluation takes too long), 0 = as
//                                        the reference does
#include <cuda.h>

#include <chrono>
#include <cstdint>
#include <cstring>
#include <vector>

#include "circle.hpp"

namespace {

using orc::CircleCoset;
using orc::M31;

CUcontext g_ctx = nullptr;
CUmodule g_mod = nullptr;
CUfunction g_interleave = nullptr, g_layer = nullptr, g_bitrev = nullptr, g_deinterleave = nullptr;
bool g_fast_twiddles = false;

unsigned grid_for(size_t count) { return (unsigned)((count + 255) / 256); }

struct DevMem {
  CUdeviceptr p = 0;
  explicit DevMem(size_t bytes) {
    if (cuMemAlloc(&p, bytes) != CUDA_SUCCESS) p = 0;
  }
  ~DevMem() {
    if (p) cuMemFree(p);
  }
};

int launch(CUfunction f, size_t count, void** args) {
  return cuLaunchKernel(f, grid_for(count), 1, 1, 256, 1, 1, 0, nullptr, args, nullptr) == CUDA_SUCCESS ? 0 : -5;
}

// circle.zig:65-82 via the oracle's restatement (faithful: per-point `at`).
std::vector<uint32_t> twiddle_tree(unsigned lg) {
  const CircleCoset half = CircleCoset::canonicHalf(lg);
  const std::vector<M31> tw = orc::precomputeTwiddles(half, !g_fast_twiddles);
  std::vector<uint32_t> out(tw.size());
  for (size_t k = 0; k < tw.size(); ++k) out[k] = tw[k].v;
  return out;
}

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

struct EventPair {
  CUevent a = nullptr, b = nullptr;
  EventPair() {
    cuEventCreate(&a, CU_EVENT_DEFAULT);
    cuEventCreate(&b, CU_EVENT_DEFAULT);
  }
  ~EventPair() {
    if (a) cuEventDestroy(a);
    if (b) cuEventDestroy(b);
  }
  float ms() {
    float v = 0;
    cuEventSynchronize(b);
    cuEventElapsedTime(&v, a, b);
    return v;
  }
};

}  // namespace

extern "C" int ref_cfft_init(const char* cubin_path) {
  if (g_mod) return 0;
  CUdevice dev;
  if (cuInit(0) != CUDA_SUCCESS || cuDeviceGet(&dev, 0) != CUDA_SUCCESS) return -5;
  if (cuDevicePrimaryCtxRetain(&g_ctx, dev) != CUDA_SUCCESS) return -5;
  if (cuCtxSetCurrent(g_ctx) != CUDA_SUCCESS) return -5;
  if (cuModuleLoad(&g_mod, cubin_path) != CUDA_SUCCESS) return -5;
  if (cuModuleGetFunction(&g_interleave, g_mod, "circle_interleave") != CUDA_SUCCESS ||
      cuModuleGetFunction(&g_layer, g_mod, "circle_fft_layer") != CUDA_SUCCESS ||
      cuModuleGetFunction(&g_bitrev, g_mod, "circle_bitreverse") != CUDA_SUCCESS ||
      cuModuleGetFunction(&g_deinterleave, g_mod, "circle_deinterleave") != CUDA_SUCCESS)
    return -5;
  return 0;
}

extern "C" void ref_cfft_twiddles(int fast) { g_fast_twiddles = fast != 0; }

// circlefft_gpu.zig:46-105. Sizes below lg = 3 fall back to the CPU there; they are
// rejected here (the bar is only timed at lg >= 3).
extern "C" int ref_cfft_fft(const uint32_t* coeffs, uint32_t* evals, unsigned lg, double* t) {
  if (!g_mod || lg < 3 || lg > 28) return -1;
  if (cuCtxSetCurrent(g_ctx) != CUDA_SUCCESS) return -5;
  const auto t0 = std::chrono::steady_clock::now();
  const size_t n = (size_t)1 << lg, half = n / 2;
  DevMem d_coeffs(n * 4), d_values(n * 4), d_tree(half * 4), d_circle(half * 4);
  if (!d_coeffs.p || !d_values.p || !d_tree.p || !d_circle.p) return -3;
  if (cuMemcpyHtoD(d_coeffs.p, coeffs, n * 4) != CUDA_SUCCESS) return -5;
  const std::vector<uint32_t> tw = twiddle_tree(lg);
  if (cuMemcpyHtoD(d_tree.p, tw.data(), half * 4) != CUDA_SUCCESS) return -5;
  std::vector<M31> tw_m(tw.size());
  for (size_t k = 0; k < tw.size(); ++k) tw_m[k] = M31(tw[k]);
  const size_t first_len = orc::lineTwiddleLen(0, lg);
  const std::vector<M31> ctw = orc::circleTwiddles(tw_m.data() + orc::lineTwiddleOffset(tw.size(), 0, lg), first_len);
  if (cuMemcpyHtoD(d_circle.p, ctw.data(), half * 4) != CUDA_SUCCESS) return -5;
  EventPair ev;
  cuEventRecord(ev.a, nullptr);
  uint32_t half32 = (uint32_t)half, n32 = (uint32_t)n, zero = 0;
  int rc = 0;
  {
    void* a[] = {&d_coeffs.p, &d_values.p, &half32};
    rc |= launch(g_interleave, half, a);
  }
  for (uint32_t i = lg - 1; i >= 1; --i) {  // line layers, largest to smallest
    const size_t len = orc::lineTwiddleLen(i - 1, lg);
    CUdeviceptr d_tw = d_tree.p + (CUdeviceptr)(orc::lineTwiddleOffset(tw.size(), i - 1, lg) * 4);
    void* a[] = {&d_values.p, &d_tw, &n32, &i, &zero};
    rc |= launch(g_layer, len << i, a);
  }
  {
    uint32_t layer0 = 0;
    void* a[] = {&d_values.p, &d_circle.p, &n32, &layer0, &zero};
    rc |= launch(g_layer, half, a);
  }
  {
    void* a[] = {&d_values.p, &n32};
    rc |= launch(g_bitrev, n, a);
  }
  cuEventRecord(ev.b, nullptr);
  if (cuMemcpyDtoH(evals, d_values.p, n * 4) != CUDA_SUCCESS) rc = -5;
  const float dev_ms = ev.ms();
  if (t) t[0] = ms_since(t0), t[1] = dev_ms;
  return rc;
}

// circlefft_gpu.zig:108-175.
extern "C" int ref_cfft_ifft(const uint32_t* evals, uint32_t* coeffs, unsigned lg, double* t) {
  if (!g_mod || lg < 3 || lg > 28) return -1;
  if (cuCtxSetCurrent(g_ctx) != CUDA_SUCCESS) return -5;
  const auto t0 = std::chrono::steady_clock::now();
  const size_t n = (size_t)1 << lg, half = n / 2;
  DevMem d_values(n * 4), d_coeffs(n * 4), d_tree(half * 4), d_circle(half * 4);
  if (!d_coeffs.p || !d_values.p || !d_tree.p || !d_circle.p) return -3;
  if (cuMemcpyHtoD(d_values.p, evals, n * 4) != CUDA_SUCCESS) return -5;
  std::vector<uint32_t> tw = twiddle_tree(lg);
  std::vector<M31> tw_m(tw.size());
  for (size_t k = 0; k < tw.size(); ++k) tw_m[k] = M31(tw[k]).inv(), tw[k] = tw_m[k].v;
  if (cuMemcpyHtoD(d_tree.p, tw.data(), half * 4) != CUDA_SUCCESS) return -5;
  const size_t first_len = orc::lineTwiddleLen(0, lg);
  const std::vector<M31> ctw = orc::circleTwiddles(tw_m.data() + orc::lineTwiddleOffset(tw.size(), 0, lg), first_len);
  if (cuMemcpyHtoD(d_circle.p, ctw.data(), half * 4) != CUDA_SUCCESS) return -5;
  EventPair ev;
  cuEventRecord(ev.a, nullptr);
  uint32_t half32 = (uint32_t)half, n32 = (uint32_t)n, one = 1;
  int rc = 0;
  {
    void* a[] = {&d_values.p, &n32};
    rc |= launch(g_bitrev, n, a);
  }
  {
    uint32_t layer0 = 0;
    void* a[] = {&d_values.p, &d_circle.p, &n32, &layer0, &one};
    rc |= launch(g_layer, half, a);
  }
  for (uint32_t i = 1; i <= lg - 1; ++i) {  // line layers, smallest to largest
    const size_t len = orc::lineTwiddleLen(i - 1, lg);
    CUdeviceptr d_tw = d_tree.p + (CUdeviceptr)(orc::lineTwiddleOffset(tw.size(), i - 1, lg) * 4);
    void* a[] = {&d_values.p, &d_tw, &n32, &i, &one};
    rc |= launch(g_layer, len << i, a);
  }
  {
    uint32_t inv_n = M31::fromInt((uint32_t)n).inv().v;
    void* a[] = {&d_values.p, &d_coeffs.p, &half32, &inv_n};
    rc |= launch(g_deinterleave, half, a);
  }
  cuEventRecord(ev.b, nullptr);
  if (cuMemcpyDtoH(coeffs, d_coeffs.p, n * 4) != CUDA_SUCCESS) rc = -5;
  const float dev_ms = ev.ms();
  if (t) t[0] = ms_since(t0), t[1] = dev_ms;
  return rc;
}
