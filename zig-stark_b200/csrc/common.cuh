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

}  // namespace zs
