// GenericStark(Air) prover on the device (see stark.cu).
#pragma once
#include <vector>

#include "common.cuh"

namespace zs {

// Proves `trace` (and `preprocessed`) for the compiled-in AIR `air_id` with the
// transcript separator `sep`; every argument is in the reference's wire format.
// Returns the serialized GenericStark(Air).Proof (stark.zig:107-122).
std::vector<uint8_t> stark_prove(uint32_t air_id, const uint8_t* params, size_t params_len, const uint8_t* pi,
                                 size_t pi_len, const uint8_t* pre, size_t pre_len, const uint8_t* trace,
                                 size_t trace_len, const uint8_t* sep, size_t sep_len, cudaStream_t st);

// Per-column commitment roots (stark.zig:397-414) as a wire []Digest.
std::vector<uint8_t> commit_columns(const uint8_t* cols, size_t cols_len, unsigned trace_log, unsigned log_blowup,
                                    cudaStream_t st);

}  // namespace zs
