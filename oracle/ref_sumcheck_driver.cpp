// ORACLE — test and benchmark infrastructure only. Host side of the reference's own GPU
// sum-check round kernels (src/cuda/kernels/sumcheck.cu: sumcheck_values and
// sumcheck_values128, compiled from the reference's source for sm_100a by
// oracle/build_ref.sh into oracle/_ref/), so that they can be checked against the oracle
// and timed beside this library's kernels on the same B200.
//
// This restates src/cuda/sumcheck_gpu.zig:36-151 call for call: per call it allocates
// the five device buffers, copies the tables, coefficients, indices, offsets and a zeroed
// packed-values array to the device, launches one thread per `rest` (256 threads per
// block), synchronizes, copies the packed values back and unpacks them. The reference
// creates its own context (src/cuda/cuda.zig); this driver uses the device's primary
// context so it can share a process with the CUDA runtime.
//
// Exported (extern "C"):
//   ref_sc_init(cubin_path)                      load the module; 0 on success
//   ref_sc_values(wide, cur, len, m, coeffs, nterms, indices, n_indices, offsets, dmax,
//                 half, out, t)                  one round; t[0] = wall ms of the call,
//                                                t[1] = device ms of its launch
// Inputs the kernels' 32-bit index arithmetic cannot address (m * len >= 2^32, or 2^31
// elements of 16 bytes), half = 0 (an empty grid) and malformed terms return -2 without
// a launch.
#include <cuda.h>

#include <chrono>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

CUcontext g_ctx = nullptr;
CUmodule g_mod = nullptr;
CUfunction g_v8 = nullptr, g_v128 = nullptr;

struct DevMem {
  CUdeviceptr p = 0;
  explicit DevMem(size_t bytes) {
    if (cuMemAlloc(&p, bytes ? bytes : 4) != CUDA_SUCCESS) p = 0;
  }
  ~DevMem() {
    if (p) cuMemFree(p);
  }
};

}  // namespace

extern "C" int ref_sc_init(const char* cubin_path) {
  if (g_mod) return 0;
  CUdevice dev;
  if (cuInit(0) != CUDA_SUCCESS || cuDeviceGet(&dev, 0) != CUDA_SUCCESS) return -5;
  if (cuDevicePrimaryCtxRetain(&g_ctx, dev) != CUDA_SUCCESS) return -5;
  if (cuCtxSetCurrent(g_ctx) != CUDA_SUCCESS) return -5;
  if (cuModuleLoad(&g_mod, cubin_path) != CUDA_SUCCESS) return -5;
  if (cuModuleGetFunction(&g_v8, g_mod, "sumcheck_values") != CUDA_SUCCESS ||
      cuModuleGetFunction(&g_v128, g_mod, "sumcheck_values128") != CUDA_SUCCESS)
    return -5;
  return 0;
}

extern "C" int ref_sc_values(int wide, const uint8_t* cur, size_t len, size_t m, const uint8_t* coeffs,
                             size_t nterms, const uint32_t* indices, size_t n_indices, const uint32_t* offsets,
                             size_t dmax, size_t half, uint8_t* out, double* t) {
  if (!g_mod) return -1;
  const size_t es = wide ? 16 : 1;
  if (half == 0 || 2 * half > len || m * len * (wide ? 2 : 1) >= ((size_t)1 << 32) || dmax > 255) return -2;
  if (offsets[0] != 0 || offsets[nterms] != n_indices) return -2;
  for (size_t k = 0; k < nterms; ++k)
    if (offsets[k + 1] < offsets[k]) return -2;
  for (size_t j = 0; j < n_indices; ++j)
    if (indices[j] >= m) return -2;
  if (cuCtxSetCurrent(g_ctx) != CUDA_SUCCESS) return -5;
  const auto t0 = std::chrono::steady_clock::now();
  const size_t words = wide ? (dmax + 1) * 4 : (dmax + 4) / 4;
  DevMem d_cur(m * len * es), d_coeffs(nterms * es), d_idx(n_indices * 4), d_off((nterms + 1) * 4), d_vals(words * 4);
  if (!d_cur.p || !d_coeffs.p || !d_idx.p || !d_off.p || !d_vals.p) return -3;
  std::vector<uint32_t> packed(words, 0);
  if (cuMemcpyHtoD(d_cur.p, cur, m * len * es) != CUDA_SUCCESS ||
      cuMemcpyHtoD(d_coeffs.p, coeffs, nterms * es) != CUDA_SUCCESS ||
      (n_indices && cuMemcpyHtoD(d_idx.p, indices, n_indices * 4) != CUDA_SUCCESS) ||
      cuMemcpyHtoD(d_off.p, offsets, (nterms + 1) * 4) != CUDA_SUCCESS ||
      cuMemcpyHtoD(d_vals.p, packed.data(), words * 4) != CUDA_SUCCESS)
    return -5;
  unsigned len32 = (unsigned)len, m32 = (unsigned)m, nterms32 = (unsigned)nterms, half32 = (unsigned)half,
           dmax32 = (unsigned)dmax;
  void* args[] = {&d_cur.p, &len32, &m32, &d_coeffs.p, &d_idx.p, &d_off.p, &nterms32, &half32, &dmax32, &d_vals.p};
  CUevent ea = nullptr, eb = nullptr;
  cuEventCreate(&ea, CU_EVENT_DEFAULT);
  cuEventCreate(&eb, CU_EVENT_DEFAULT);
  cuEventRecord(ea, nullptr);
  const CUresult lr = cuLaunchKernel(wide ? g_v128 : g_v8, (unsigned)((half + 255) / 256), 1, 1, 256, 1, 1, 0,
                                     nullptr, args, nullptr);
  cuEventRecord(eb, nullptr);
  const CUresult sr = cuCtxSynchronize();
  float dev_ms = 0;
  cuEventElapsedTime(&dev_ms, ea, eb);
  cuEventDestroy(ea);
  cuEventDestroy(eb);
  if (lr != CUDA_SUCCESS || sr != CUDA_SUCCESS) return -5;
  if (cuMemcpyDtoH(packed.data(), d_vals.p, words * 4) != CUDA_SUCCESS) return -5;
  if (wide) {
    std::memcpy(out, packed.data(), (dmax + 1) * 16);
  } else {
    for (size_t i = 0; i <= dmax; ++i) out[i] = (uint8_t)(packed[i >> 2] >> (8 * (i & 3)));
  }
  if (t) {
    t[0] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    t[1] = dev_ms;
  }
  return 0;
}
