// Circle low-degree extension for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: a plugin inside a host process that reserves
// all device memory up front in its own arena and forbids later allocations, or a
// latency-bound loop in which an allocation (which can synchronize the device) is not
// acceptable. zs_m31_circle_lde_noalloc serves them: it takes the caller's device
// input and output buffers and keeps everything else it needs -- the twiddle tables
// of both domains and the transform's intermediate passes -- in one file-scope device
// array of fixed size, so it never allocates.
//
// Costs and limits, stated for users of this entry point:
//   - every GPU on which this library's device code is loaded holds the array (16 MiB)
//     until the process exits. Under CUDA's default lazy module loading that happens
//     on the first call on the device (the address lookup below), not when the library
//     is opened, so a caller that later reserves all free device memory makes one small
//     call first (or sets CUDA_MODULE_LOADING=EAGER);
//   - a call needs 2*2^L + 2*2^(L+B) + C*(2^L + 2^(L+B)) words of it, at most
//     kNoallocWords (2^22 words); larger requests are rejected with -2;
//   - all calls share the array and it keeps the last call's contents, so calls
//     whose work overlaps on the GPU (different streams, or several host threads)
//     race and must be serialized by the caller. Nothing in the array has to start
//     at zero: every word a call reads was written earlier in the same call;
//   - the first call on a device looks up the array's device address (once per
//     device, with that device current); make that first call before any stream
//     capture begins. The address is kept for the life of the process: after a
//     cudaDeviceReset the module is reloaded elsewhere, so the entry point must not be
//     used across a device reset.
#include <mutex>

#include "../../include/zs_m31.h"
#include "circle.cuh"

namespace zs {
namespace {

constexpr size_t kNoallocWords = (size_t)1 << 22;  // 16 MiB
constexpr int kMaxDevices = 64;

static __device__ __align__(256) uint32_t g_lde_scratch[kNoallocWords];

std::mutex g_setup_mutex;
uint32_t* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_lde_scratch on the current device (looked up once per device).
int32_t scratch_for_current_device(uint32_t** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return ZS_EDEVICE;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    uint32_t* ptr = nullptr;
    if (cudaGetSymbolAddress((void**)&ptr, g_lde_scratch) != cudaSuccess || !ptr) return ZS_EDEVICE;
    g_scratch_ptr[dev] = ptr;
  }
  *out = g_scratch_ptr[dev];
  return ZS_OK;
}

}  // namespace
}  // namespace zs

using namespace zs;

extern "C" int32_t zs_m31_circle_lde_noalloc(const uint32_t* d_in, uint32_t* d_out, uint32_t n_columns,
                                             uint32_t log_rows, uint32_t log_blowup, void* stream) {
  if (!d_in || !d_out || n_columns == 0) return ZS_EMALFORMED;
  if (log_rows < 1 || log_rows + log_blowup > 28) return ZS_EMALFORMED;
  const size_t n = (size_t)1 << log_rows, N = (size_t)1 << (log_rows + log_blowup);
  const size_t need = 2 * n + 2 * N + (size_t)n_columns * (n + N);
  if (need > kNoallocWords) return ZS_EMALFORMED;
  uint32_t* base = nullptr;
  const int32_t rc = scratch_for_current_device(&base);
  if (rc != ZS_OK) return rc;
  uint32_t* tw_small = base;
  uint32_t* itw_small = tw_small + n;
  uint32_t* tw_big = itw_small + n;
  uint32_t* itw_big = tw_big + N;
  uint32_t* work = itw_big + N;
  cudaStream_t st = (cudaStream_t)stream;
  try {
    circle_twiddles_into(log_rows, tw_small, itw_small, st);
    circle_twiddles_into(log_rows + log_blowup, tw_big, itw_big, st);
    circle_lde_tables(d_in, n, d_out, N, n_columns, log_rows, log_blowup, itw_small, tw_big, work, st);
  } catch (const Error& e) {
    return e.code;
  } catch (...) {
    return ZS_EGENERIC;
  }
  return ZS_OK;
}
