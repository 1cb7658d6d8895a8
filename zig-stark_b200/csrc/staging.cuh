// Host -> device uploads of caller memory through pinned staging buffers.
//
// The inputs of a proof arrive in pageable host memory (a wire-format trace). A
// pageable cudaMemcpyAsync is staged by the driver on the calling thread at the
// speed of one memcpy; here the staging copy is split across a small pool of host
// threads and double-buffered against the DMA of the previous chunk, so an upload
// runs at the PCIe rate instead of one core's memcpy rate.
#pragma once
#include <cstddef>

#include "common.cuh"

namespace zs {

// Copies `bytes` from host memory `src` to device memory `dst` in stream order on
// `st`. Returns once `src` may be reused; the device copy completes in stream order.
void upload_bytes(void* dst, const void* src, size_t bytes, cudaStream_t st);

// memcpy of host memory, split over the host copy pool when it is large (a served
// request's copy of a 2^22-row trace is most of a gigabyte) and the pool is free; on the
// calling thread otherwise.
void host_copy(void* dst, const void* src, size_t bytes);

// Uploads the low 32-bit word of every 16-byte element of C columns (column j: n
// elements at cols[j]) to dst (column j at dst + j * n), packing on the host so a
// QM31-embedded M31 column crosses PCIe at a quarter of its wire size. high[j] is set
// when some element of column j has a non-zero word among its upper three (that
// column's packed words are then incomplete and the caller uploads it whole).
void upload_low_words(uint32_t* dst, const uint8_t* const* cols, uint32_t C, size_t n, uint8_t* high,
                      cudaStream_t st);

// The calling thread's uploads wait for the host copy pool while the scope lives,
// instead of packing on their own thread when another prover holds the pool. A large
// proof sets it, so its upload keeps the pool's bandwidth while small proofs share the
// device with it (their short copies run on their own threads meanwhile).
class UploadPriority {
 public:
  explicit UploadPriority(bool high);
  ~UploadPriority();
  UploadPriority(const UploadPriority&) = delete;
  UploadPriority& operator=(const UploadPriority&) = delete;

 private:
  bool prev_;
};

// The small transfers of a proof (constants, roots, evaluations, query reveals) go
// through pinned memory too: a pageable copy takes the driver's staging path, on which
// concurrent provers would queue behind one another's uploads.
//
// A PinnedScope binds a slot of pinned memory (upload buffers and a bump arena for
// small transfers) to the calling thread for one proof. Slots come from a
// process-wide bank and go back to it, never freed, so threads that prove once do not
// pin host memory each time. Every copy through the slot is issued on `st`, which the
// scope drains before it returns the slot (also when a proof fails part-way). Without
// a scope the calls below fall back to pageable copies.
class PinnedScope {
 public:
  explicit PinnedScope(cudaStream_t st);
  ~PinnedScope();
  PinnedScope(const PinnedScope&) = delete;
  PinnedScope& operator=(const PinnedScope&) = delete;

 private:
  cudaStream_t st_;
  void* slot_;
  void* prev_;
};
// Host -> device through a fresh pinned region (stream ordered; `src` reusable at return).
void h2d_small(void* dst, const void* src, size_t bytes, cudaStream_t st);
// Device -> host through a fresh pinned region; synchronizes `st`.
void d2h_small(void* dst, const void* src, size_t bytes, cudaStream_t st);
// Several device -> host copies with one wait on `st`.
struct D2H {
  void* dst;
  const void* src;
  size_t bytes;
};
void d2h_many(const D2H* copies, size_t count, cudaStream_t st);

}  // namespace zs
