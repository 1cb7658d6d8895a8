// Shared host/device helpers: status codes, CUDA error propagation, bit tricks.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <stdexcept>
#include <string>

#include "field.cuh"

namespace zs {

// Return codes of the C ABI (zig-capi.h:20-21 plus -5 for device failures).
enum Status : int32_t {
  ZS_OK = 0,
  ZS_EGENERIC = -1,
  ZS_EMALFORMED = -2,
  ZS_ENOMEM = -3,
  ZS_EPROTOCOL = -4,
  ZS_EDEVICE = -5,
};

struct Error : std::runtime_error {
  int32_t code;
  Error(int32_t c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    int32_t code = e == cudaErrorMemoryAllocation ? ZS_ENOMEM : ZS_EDEVICE;
    throw Error(code, std::string(what) + ": " + cudaGetErrorString(e));
  }
}
#define ZS_CUDA(x) ::zs::cuda_check((x), #x)

// Reverses the low `bits` bits of x (bits <= 32).
ZS_HD uint32_t bitrev(uint32_t x, unsigned bits) {
  if (bits == 0) return 0;
#ifdef __CUDA_ARCH__
  return __brev(x) >> (32 - bits);
#else
  uint32_t r = 0;
  for (unsigned b = 0; b < bits; ++b) r |= ((x >> b) & 1u) << (bits - 1 - b);
  return r;
#endif
}

// Freed blocks stay in the device's stream-ordered pool instead of going back to the
// driver at every synchronization, so repeated proofs do not map their memory again.
inline void retain_pool_memory() {
  static std::mutex mu;
  static uint64_t done = 0;
  int dev = 0;
  ZS_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if (dev < 64 && (done >> dev & 1)) return;
  cudaMemPool_t pool;
  ZS_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
  uint64_t keep = UINT64_MAX;
  ZS_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
  // A block freed on one prover's stream is reused by another only once the free has
  // completed: the pool never makes one proof's stream wait on another's.
  int no = 0;
  ZS_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &no));
  if (dev < 64) done |= 1ull << dev;
}


// Non-blocking streams owned by the calling thread, created on first use per device and
// slot and kept for the thread's life (creating and destroying streams and events costs
// tens of microseconds per proof otherwise). Slots: 0 the stream of a zs_m31_prove call,
// 1 and 2 a proof's upload and tree side streams. `ev` is an event for the slot's use.
struct ThreadStreams {
  static constexpr int kDevices = 64, kSlots = 3;
  cudaStream_t s[kDevices][kSlots] = {};
  cudaEvent_t ev[kDevices][kSlots] = {};
  ~ThreadStreams() {
    for (int d = 0; d < kDevices; ++d)
      for (int k = 0; k < kSlots; ++k) {
        if (ev[d][k]) cudaEventDestroy(ev[d][k]);
        if (s[d][k]) cudaStreamDestroy(s[d][k]);
      }
  }
};
inline void thread_stream(int slot, cudaStream_t* st, cudaEvent_t* ev = nullptr) {
  static thread_local ThreadStreams ts;
  int dev = 0;
  cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= ThreadStreams::kDevices || slot < 0 || slot >= ThreadStreams::kSlots)
    throw Error(ZS_EDEVICE, "thread stream slot");
  if (!ts.s[dev][slot]) {
    cuda_check(cudaStreamCreateWithFlags(&ts.s[dev][slot], cudaStreamNonBlocking), "cudaStreamCreateWithFlags");
    cuda_check(cudaEventCreateWithFlags(&ts.ev[dev][slot], cudaEventDisableTiming), "cudaEventCreateWithFlags");
  }
  *st = ts.s[dev][slot];
  if (ev) *ev = ts.ev[dev][slot];
}
}  // namespace zs
