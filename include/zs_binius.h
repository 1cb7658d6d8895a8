/* C ABI of the Binius sum-check on the B200 (sm_100a).
 *
 * The reference's Binius prover computes each sum-check round's evaluations
 *   values[t] = sum_rest sum_terms coeff * prod_f (a_f + t (a_f + b_f)),  t = 0..dmax,
 * on the CPU (src/binius/sumcheck.zig:357-372) or through an accelerator hook
 * (src/binius/accel.zig:9-47) that its CUDA port implements (src/cuda/sumcheck_gpu.zig:36-151,
 * kernels src/cuda/kernels/sumcheck.cu). The first two entry points are that hook: the
 * same flattened inputs, the same bytes out, so a Zig caller registers them as
 * accel.gf256_values / accel.gf128_values through a two-line wrapper. The device entry
 * points below them keep the tables in device memory between rounds, and
 * zs_binius_sumcheck_prove_combination runs Sumcheck(F).proveCombination
 * (src/binius/sumcheck.zig:208-395) on them end to end.
 *
 * Fields: TowerField(3) = GF(2^8) (one byte per element) and TowerField(7) = GF(2^128)
 * (16 little-endian bytes per element) of src/binius/tower.zig; field_bits is 8 or 128.
 * Terms: term k has coefficient coeffs[k] and the factor tables
 * indices[offsets[k] .. offsets[k + 1]) (offsets: nterms + 1 entries, offsets[0] = 0,
 * non-decreasing, offsets[nterms] = n_indices); 1 <= nterms <= 256, n_indices <= 1024,
 * every index < m <= 65535. Table f's element i is at (f * len + i) * element size.
 * Conventions as zs_m31.h: 0 on success, -2 for malformed arguments (nothing launched),
 * -3 out of device memory, -5 other device errors; `stream` is a cudaStream_t (NULL: the
 * default stream). */
#ifndef ZS_BINIUS_H
#define ZS_BINIUS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* accel.Gf256ValuesFn (src/binius/accel.zig:9-26) as sumcheck_gpu.computeValues computes
 * it (src/cuda/sumcheck_gpu.zig:36-93): cur_flat holds m tables of len bytes (host
 * memory), rows (2 rest, 2 rest + 1) for rest < half (2 half <= len); out receives
 * dmax + 1 bytes, values[t] for t = 0..dmax (dmax <= 255). Synchronous. */
int32_t zs_binius_sumcheck_values_gf256(const uint8_t *cur_flat, size_t len, size_t m, const uint8_t *coeffs,
                                        size_t nterms, const uint32_t *indices, size_t n_indices,
                                        const uint32_t *offsets, size_t dmax, size_t half, uint8_t *out,
                                        void *stream);

/* accel.Gf128ValuesFn (src/binius/accel.zig:43-47) as sumcheck_gpu.computeValues128
 * computes it (src/cuda/sumcheck_gpu.zig:95-151): every element 16 bytes (cur_flat
 * m * len * 16 bytes, coeffs nterms * 16, out (dmax + 1) * 16); otherwise as above. */
int32_t zs_binius_sumcheck_values_gf128(const uint8_t *cur_flat, size_t len, size_t m, const uint8_t *coeffs,
                                        size_t nterms, const uint32_t *indices, size_t n_indices,
                                        const uint32_t *offsets, size_t dmax, size_t half, uint8_t *out,
                                        void *stream);

/* The same round on tables already in device memory (d_cur; 16-byte aligned for
 * field_bits 128), asynchronous on `stream`. d_out (device, 4-byte aligned) receives the
 * values as the hook returns them, in (dmax + 4) / 4 * 4 bytes for field_bits 8 and
 * (dmax + 1) * 16 bytes for 128. The term arrays are host memory, read before the call
 * returns. */
int32_t zs_binius_sumcheck_values_device(uint32_t field_bits, const void *d_cur, size_t len, size_t m,
                                         const uint8_t *coeffs, size_t nterms, const uint32_t *indices,
                                         size_t n_indices, const uint32_t *offsets, size_t dmax, size_t half,
                                         void *d_out, void *stream);

/* The table fold of a round (src/binius/sumcheck.zig:379-388) on device tables:
 * d_next[f * (len / 2) + rest] = a + r (a + b), a = d_cur[f * len + 2 rest],
 * b = d_cur[f * len + 2 rest + 1], for f < m. r: one element in host memory (1 or 16
 * bytes). d_scratch: 64 KB of device memory for field_bits 128 (the multiply table of r),
 * unused for 8. Asynchronous on `stream`; d_next must not overlap d_cur. */
int32_t zs_binius_sumcheck_fold_device(uint32_t field_bits, const void *d_cur, size_t len, size_t m,
                                       const uint8_t *r, void *d_next, void *d_scratch, void *stream);

/* Sumcheck(F).proveCombination (src/binius/sumcheck.zig:208-395) with its optional
 * transcript seed (Transcript.initBytes(seed) when has_seed is set, else
 * Transcript.init(claimed sum)): m tables of 2^k elements (host memory, m * 2^k element
 * sizes), copied to the device once; every round (values, interpolation, the SHA-256
 * transcript step, fold) runs on the device, and the host waits once, for the proof.
 * claimed_out: one element (the hypercube sum). rounds_out: k * (dmax + 1) elements, round
 * i's low-first coefficients at i * (dmax + 1), dmax = the longest term (dmax + 1 <= 64).
 * Synchronous. */
int32_t zs_binius_sumcheck_prove_combination(uint32_t field_bits, const uint8_t *tables, size_t k, size_t m,
                                             const uint8_t *coeffs, size_t nterms, const uint32_t *indices,
                                             size_t n_indices, const uint32_t *offsets, const uint8_t *seed,
                                             size_t seed_len, int32_t has_seed, uint8_t *claimed_out,
                                             uint8_t *rounds_out, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* ZS_BINIUS_H */
