// Host-side GenericStark verifier (see verify.cu).
#pragma once
#include "common.cuh"

namespace zs {

// True when `proof` (wire GenericStark(Air).Proof) verifies for the AIR, params,
// public inputs and channel separator; throws Error(-2) on malformed input.
bool stark_verify(uint32_t air_id, const uint8_t* params, size_t params_len, const uint8_t* pi, size_t pi_len,
                  const uint8_t* proof, size_t proof_len, const uint8_t* sep, size_t sep_len);

}  // namespace zs
