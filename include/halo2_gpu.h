/*
 * halo2_gpu.h -- C ABI of the B200 (sm_100a) BN254 Halo2/KZG prover hot path.
 *
 * Drop-in for the reference's static library `libhalo2_gpu`: every `_halo2_*`
 * symbol below keeps the name, argument order, argument meaning and error
 * behaviour of the reference launcher it replaces (cited per entry, paths
 * relative to the axiom-crypto/halo2-gpu tree).  The Rust crate binds them in
 * halo2_proofs/src/cuda/culib.rs:28-652 and
 * halo2_proofs/src/plonk/evaluation.rs:1434-1568.
 *
 * Conventions (halo2_proofs/cuda/include/common/halo2_ffi.h:1-62):
 *  - Field elements are 32-byte Montgomery-form BN254 Fr/Fq, little-endian
 *    64-bit limbs (the halo2curves memory image).  G1 affine points are 64
 *    bytes {x, y}, infinity = (0, 0).  MSM results are the 96-byte Jacobian
 *    image {X, Y, Z} with Z = 1, or (0, 1, 0) for infinity.
 *  - `void*` arguments named d_* are device pointers; FFITraitObject carries a
 *    host or device address as documented per entry.
 *  - `scratch` is caller-owned device memory of at least the matching
 *    `_workspace_size` bytes (256-byte aligned is best).  Launchers never
 *    allocate device memory.
 *  - Work is enqueued on `stream`; entries with host outputs synchronise the
 *    stream before returning, device-output entries do not.
 *  - RustError.code == 0 on success; otherwise a cudaError_t value or a
 *    reference-compatible sentinel (-1 / 2 / -6 for unsupported NTT types).
 *    A non-null RustError.message is heap memory owned by the caller (free()).
 */
#ifndef HALO2_GPU_H
#define HALO2_GPU_H

#include <stdbool.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct RustError {
    int code;
    char* message;
} RustError;

typedef struct FFITraitObject {
    uint64_t* ptr;
} FFITraitObject;

typedef void* h2b_stream_t; /* cudaStream_t */

/* ------------------------------------------------------------------ MSM --- */

/* culib.rs:30 ; multiexp.cu:183-188 */
uint64_t _halo2_msm_max_length(uint64_t free_bytes);
/* culib.rs:32 ; multiexp.cu:191-195 */
uint64_t _halo2_multiexp_workspace_size(uint64_t length);
/* culib.rs:34-43 ; multiexp.cu:260-327 -- host scalars, host bases, host out */
RustError _halo2_multiexp(const FFITraitObject* scalar, const FFITraitObject* point, const FFITraitObject* output,
                          uint64_t length, void* scratch, uint64_t scratch_bytes, h2b_stream_t stream);
/* culib.rs:45 ; multiexp.cu:333-337 */
uint64_t _halo2_multiexp_device_bases_workspace_size(uint64_t length);
/* culib.rs:47-56 ; multiexp.cu:346-412 -- host scalars, device bases, host out */
RustError _halo2_multiexp_device_bases(const FFITraitObject* h_scalar, const void* d_bases,
                                       const FFITraitObject* h_output, uint64_t length, void* scratch,
                                       uint64_t scratch_bytes, h2b_stream_t stream);
/* culib.rs:58 ; multiexp.cu:419-423 */
uint64_t _halo2_multiexp_device_scalars_device_bases_workspace_size(uint64_t length);
/* culib.rs:60-70 ; multiexp.cu:436-525 -- device scalars (not mutated), device bases, host out */
RustError _halo2_multiexp_device_scalars_device_bases(const void* d_scalar, const void* d_bases,
                                                      const FFITraitObject* h_output, uint64_t length,
                                                      void* scratch, uint64_t scratch_bytes, h2b_stream_t stream);

/* ------------------------------------------------------------- batch inv --- */

/* culib.rs:72-79 ; polynomial/operations.cu:16-42 -- in place, zeros stay zero, field_type 0 = Fr, 1 = Fq */
RustError _halo2_batch_invert(void* d_data, uint32_t field_type, uint64_t length, h2b_stream_t stream);

/* ---------------------------------------------------- products and scans --- */

/* culib.rs:81-82 ; commitment/commit_product.cu:35-50 */
uint64_t _halo2_commit_product_max_len(uint64_t length, uint64_t free_bytes);
uint64_t _halo2_commit_product_workspace_size(uint64_t poly_length);
/* culib.rs:87-100 ; commitment/commit_product.cu:51-139 -- host polys, device beta/gamma */
RustError _halo2_commit_product(const FFITraitObject* lookup_product, const FFITraitObject* permuted_input,
                                const FFITraitObject* permuted_table, const FFITraitObject* compressed_input,
                                const FFITraitObject* compressed_table, const void* beta_device,
                                const void* gamma_device, uint64_t length, uint64_t offset, void* scratch,
                                uint64_t scratch_bytes, h2b_stream_t stream);
/* culib.rs:114-125 ; commitment/commit_product.cu:141-186 -- all device, no scratch */
RustError _halo2_commit_product_device_inputs(const FFITraitObject* d_lookup_product,
                                              const FFITraitObject* d_permuted_input,
                                              const FFITraitObject* d_permuted_table,
                                              const FFITraitObject* d_compressed_input,
                                              const FFITraitObject* d_compressed_table, const void* beta_device,
                                              const void* gamma_device, uint64_t length, uint64_t offset,
                                              h2b_stream_t stream);

/* culib.rs:143-144 ; commitment/permutation_commit.cu:37-50 */
uint64_t _halo2_permutation_product_max_len(uint64_t length, uint64_t free_bytes);
uint64_t _halo2_permutation_product_workspace_size(uint64_t poly_length);
/* culib.rs:147-162 ; commitment/permutation_commit.cu:51-146 -- host polys, device scalars */
RustError _halo2_permutation_product(const FFITraitObject* modified_values, const FFITraitObject* permutations,
                                     const FFITraitObject* values, const void* beta_device, const void* gamma_device,
                                     const void* delta_device, const void* omega_device, void* deltaomega_device,
                                     uint64_t length, uint64_t offset, uint64_t batch, void* scratch,
                                     uint64_t scratch_bytes, h2b_stream_t stream);
/* culib.rs:164 ; commitment/permutation_commit.cu:163-167 */
uint64_t _halo2_permutation_product_device_inputs_workspace_size(uint64_t poly_length);
/* culib.rs:184-199 ; commitment/permutation_commit.cu:181-256 -- all device */
RustError _halo2_permutation_product_device_inputs(const FFITraitObject* modified_values_device,
                                                   const FFITraitObject* permutations_device,
                                                   const FFITraitObject* values_device, const void* beta_device,
                                                   const void* gamma_device, const void* delta_device,
                                                   const void* omega_device, void* deltaomega_device,
                                                   uint64_t length, uint64_t offset, uint64_t batch, void* scratch,
                                                   uint64_t scratch_bytes, h2b_stream_t stream);

/* culib.rs:201-202 ; commitment/grand_product.cu:31-49 */
uint64_t _halo2_grand_product_max_len(uint64_t length, uint64_t free_bytes);
uint64_t _halo2_grand_product_workspace_size(uint64_t poly_length);
/* culib.rs:206-215 ; commitment/grand_product.cu:51-132 -- out[i] = prefix * prod_{j<=i} in[j], host polys */
RustError _halo2_grand_product(const FFITraitObject* output, const FFITraitObject* input,
                               const FFITraitObject* prefix, uint64_t poly_length, uint64_t poly_offset,
                               void* scratch, uint64_t scratch_bytes, h2b_stream_t stream);
/* culib.rs:224-230 ; commitment/grand_product.cu:139-195 -- in place on device, device prefix */
RustError _halo2_grand_product_device_inputs(const FFITraitObject* d_inout, const FFITraitObject* d_prefix,
                                             uint64_t poly_length, uint64_t poly_offset, h2b_stream_t stream);

/* ------------------------------------------------------ lookup permute --- */

/* culib.rs:127 ; commitment/permute_expression_pair.cu:185-227 */
uint64_t _halo2_permute_expression_pair_workspace_size(uint64_t n, uint64_t usable_rows);
/* culib.rs:131-141 ; commitment/permute_expression_pair.cu:229-350 -- device in/out */
RustError _halo2_permute_expression_pair(const void* d_compressed_input, const void* d_compressed_table,
                                         void* d_permuted_input, void* d_permuted_table, uint64_t n,
                                         uint64_t usable_rows, void* scratch, uint64_t scratch_bytes,
                                         h2b_stream_t stream);

/* -------------------------------------------------------- element-wise --- */

/* culib.rs:276-282 ; polynomial/polynomial.cu:420-455 */
RustError _halo2_poly_multiply_add(void* d_poly_acc, const void* d_poly_in, const void* d_scalar,
                                   uint64_t poly_length, h2b_stream_t stream);
/* culib.rs:285-291 ; polynomial/polynomial.cu:321-341 */
RustError _halo2_poly_elementwise_multiply(void* d_out, const void* d_a, const void* d_b, uint64_t length,
                                           h2b_stream_t stream);
/* culib.rs:294-298 ; polynomial/polynomial.cu:343-361 -- fills with one */
RustError _halo2_poly_fill_one(void* d_out, uint64_t length, h2b_stream_t stream);
/* culib.rs:322-328 ; polynomial/polynomial.cu:270-292 */
RustError _halo2_divide_by_vanishing_poly(void* d_poly, const void* d_t_evals, uint32_t t_len, uint64_t n,
                                          h2b_stream_t stream);
/* culib.rs:359-364 ; polynomial/polynomial.cu:363-388 */
RustError _halo2_poly_sub_short_inplace(void* d_acc, const void* d_short, uint64_t short_len, h2b_stream_t stream);
/* culib.rs:370-377 ; polynomial/polynomial.cu:390-416 */
RustError _halo2_poly_sub_short_out_of_place(void* d_out, const void* d_long, const void* d_short,
                                             uint64_t short_len, uint64_t long_len, h2b_stream_t stream);
/* culib.rs:381-385 ; polynomial/polynomial.cu:418-433 */
RustError _halo2_poly_sub_scalar_at_zero(void* d_buf, const void* d_scalar, h2b_stream_t stream);
/* culib.rs:389-395 ; polynomial/polynomial.cu:247-268 -- d_parts: device array of device pointers */
RustError _halo2_extended_from_lagrange_vec_device(void* d_out, const void* d_parts, uint32_t num_parts, uint64_t n,
                                                   h2b_stream_t stream);
/* culib.rs:399-405 ; polynomial/polynomial.cu:294-319 */
RustError _halo2_distribute_powers_zeta(void* d_a, const void* d_coset_powers, uint32_t coset_powers_len,
                                       uint64_t n, h2b_stream_t stream);

/* ------------------------------------------------- opening and witness --- */

/* culib.rs:231 ; polynomial/polynomial.cu:62-66 */
uint64_t _halo2_eval_polynomial_workspace_size(uint64_t length);
/* culib.rs:235-243 ; polynomial/polynomial.cu:68-90 -- sum_i d_poly[i] * point^i; host point; *d_result_out =
 * device address of the 32-byte result (inside scratch); does not synchronise */
RustError _halo2_eval_polynomial(const void* d_poly, const FFITraitObject* point, void** d_result_out,
                                 uint64_t length, void* scratch, uint64_t scratch_bytes, h2b_stream_t stream);
/* culib.rs:245-249 ; polynomial/polynomial.cu:135-146 */
uint64_t _halo2_eval_poly_batch_max_len(uint64_t poly_length, uint64_t batch_size, uint64_t free_bytes);
/* culib.rs:251 ; polynomial/polynomial.cu:148-154 */
uint64_t _halo2_eval_polynomial_batch_workspace_size(uint64_t poly_length, uint64_t batch_size);
/* culib.rs:254-264 ; polynomial/polynomial.cu:156-245 -- host polys (chunk [offset, offset + length), exponents
 * counted from the chunk start), host points, host results; synchronises */
RustError _halo2_eval_polynomial_batch(const FFITraitObject* poly_in_many, const FFITraitObject* eval_points,
                                       const FFITraitObject* eval_result, uint64_t poly_offset, uint64_t poly_length,
                                       uint64_t batch_size, void* scratch, uint64_t scratch_bytes,
                                       h2b_stream_t stream);
/* culib.rs:319 ; polynomial/kate_division.cu:27-36 */
uint64_t _halo2_kate_division_workspace_size(uint64_t n);
/* culib.rs:325-333 ; polynomial/kate_division.cu:47-125 -- d_q (n - 1) = (d_a - d_a(u)) / (X - u), all device */
RustError _halo2_kate_division_device(const void* d_a, void* d_q, const void* d_u, uint64_t n, void* scratch,
                                      uint64_t scratch_bytes, h2b_stream_t stream);
/* culib.rs:339-348 ; polynomial/kate_division.cu:127-250 -- quotient then zeros up to out_len */
RustError _halo2_kate_division_device_padded(const void* d_a, void* d_q, const void* d_u, uint64_t n,
                                             uint64_t out_len, void* scratch, uint64_t scratch_bytes,
                                             h2b_stream_t stream);
/* No counterpart in the reference (its batch evaluation and multiopen calculation stage HOST polynomial
 * chunks): out[i] = sum_j polys[i][j] points[i]^j for count <= 64 DEVICE polynomials of n coefficients
 * (host array of device pointers, host 32-byte points), device outputs (count x 32 B), scratch of
 * h2b_eval_many_workspace_size(n, count) bytes; one launch sequence for all, no synchronisation. */
uint64_t h2b_eval_many_workspace_size(uint64_t n, uint64_t count);
RustError h2b_eval_many_device(const void* const* d_polys, const void* points, uint64_t count, uint64_t n,
                               void* d_out, void* scratch, uint64_t scratch_bytes, h2b_stream_t stream);
/* No counterpart in the reference: acc[i] = (accumulate ? acc[i] : 0) + sum_t coeffs[t] polys[t][i] for
 * i < n, count <= 64 device polynomials (host array of device pointers, host 32-byte coefficients), one
 * pass over memory, no scratch, no synchronisation. */
RustError h2b_poly_linear_combination(void* d_acc, const void* const* d_polys, const void* coeffs, uint64_t count,
                                      uint64_t n, int accumulate, h2b_stream_t stream);
/* culib.rs:401-405 ; multiopen.cu:30-45 */
uint64_t _halo2_multiopen_poly_max_len(uint64_t poly_length, uint64_t batch_size, uint64_t free_bytes);
/* culib.rs:407-410 ; multiopen.cu:47-53 */
uint64_t _halo2_multiopen_poly_calculation_workspace_size(uint64_t poly_length, uint64_t batch_size);
/* culib.rs:414-426 ; multiopen.cu:76-175 -- host polys; evaluate_result[i] = chunk i at evaluate_point[i];
 * host poly_acc chunk = sum_i challenge_point[i] * chunk i (overwritten); synchronises */
RustError _halo2_multiopen_poly_calculation(const FFITraitObject* poly_in_many, const FFITraitObject* poly_acc,
                                            uint64_t poly_offset, uint64_t poly_length, uint64_t batch_size,
                                            const FFITraitObject* challenge_point,
                                            const FFITraitObject* evaluate_point,
                                            const FFITraitObject* evaluate_result, void* scratch,
                                            uint64_t scratch_bytes, h2b_stream_t stream);
/* culib.rs:22-26 -- the Rust-side layout of Assigned<F> records */
typedef struct AssignedLayout {
    uint32_t stride_bytes;
    uint32_t num_offset;
    uint32_t denom_offset;
} AssignedLayout;
/* culib.rs:301-308 ; polynomial/decode_assigned.cu:28-60 -- tag byte 0 Zero, 1 Trivial, 2 Rational */
RustError _halo2_decode_assigned(void* d_nums, void* d_denoms, const void* d_raw, uint64_t n, AssignedLayout layout,
                                 h2b_stream_t stream);
/* The reference's batch_invert_assigned_device (halo2_proofs/src/poly.rs:364-420: _halo2_decode_assigned per column,
 * one _halo2_batch_invert over all denominators, _halo2_poly_elementwise_multiply per column) as one entry point:
 * d_outs[c][i] = value of the Assigned<F> record i of column c (Zero 0, Trivial x, Rational n/d with d = 0 giving 0),
 * for n_cols <= 64 columns of n records each.  d_outs and d_raws are host arrays of device pointers; outputs must not
 * overlap the records.  The layout needs a 4-byte aligned stride and payload offsets inside the record (else an
 * error).  Scratch: h2b_batch_invert_assigned_workspace_size bytes. */
uint64_t h2b_batch_invert_assigned_workspace_size(uint64_t n, uint32_t n_cols);
RustError h2b_batch_invert_assigned(void* const* d_outs, const void* const* d_raws, uint32_t n_cols, uint64_t n,
                                    AssignedLayout layout, void* scratch, uint64_t scratch_bytes, h2b_stream_t stream);

/* ------------------------------------------------------------------ NTT --- */
/* ntt_type: 1 FFT, 2 iFFT, 3 cosetFFT, 4 icosetFFT, 5 unsupported, 6 CosetFFT_Part (ntt.cu:21-28);
 * for CosetFFT_Part the divisor slot carries the coset factor zeta * w_ext^j (domain.rs:527-540). */

/* culib.rs:492 ; ntt.cu:383-392 */
uint64_t _halo2_fft_normal_workspace_size(uint32_t ntt_type, uint32_t log_n, uint32_t extend_log_n);
/* culib.rs:494-504 ; ntt.cu:394-477 -- host in/out, host omega/divisor, synchronises */
RustError _halo2_fft_normal(uint32_t ntt_type, uint32_t log_n, const void* input, void* output, const void* omega,
                            const void* divisor, void* scratch, uint64_t scratch_bytes, h2b_stream_t stream);
/* culib.rs:506-511 ; ntt.cu:149-164 -- always true */
bool _halo2_fft_normal_check_memory(uint32_t ntt_type, const void* input, uint32_t log_n, uint32_t extend_log_n);
/* culib.rs:513-517 ; ntt.cu:483-490 */
uint64_t _halo2_fft_normal_to_device_workspace_size(uint32_t ntt_type, uint32_t log_n, uint32_t extend_log_n);
/* culib.rs:523-533 ; ntt.cu:510-580 -- device in/out (may alias), device omega, host divisor; FFT/iFFT/CosetFFT_Part */
RustError _halo2_fft_normal_to_device(uint32_t ntt_type, uint32_t log_n, const void* d_input, void* d_output,
                                      const void* d_omega, const void* h_divisor, void* scratch,
                                      uint64_t scratch_bytes, h2b_stream_t stream);
/* culib.rs:535-546 ; ntt.cu:584-648 -- host in (2^log_n) -> host out (2^extend_log_n), forward coset */
RustError _halo2_cosetfft(uint32_t ntt_type, uint32_t log_n, uint32_t extend_log_n, const void* input, void* output,
                          const void* omega, const void* divisor, void* scratch, uint64_t scratch_bytes,
                          h2b_stream_t stream);
/* culib.rs:548 ; ntt.cu:758-772 */
uint64_t _halo2_fft_many_workspace_size(uint32_t ntt_type, uint32_t log_n, uint32_t extend_log_n);
/* culib.rs:550-554 ; ntt.cu:777-787 */
uint64_t _halo2_fft_many_to_device_workspace_size(uint32_t ntt_type, uint32_t log_n, uint32_t extend_log_n);
/* culib.rs:561-573 ; ntt.cu:829-890 -- host arrays of host polys, device omega, host divisor */
RustError _halo2_fft_many(uint32_t ntt_type, uint32_t num_many, uint32_t log_n, uint32_t extend_log_n,
                          const FFITraitObject* input, const FFITraitObject* output, const void* omega_device,
                          const FFITraitObject* divisor, void* scratch, uint64_t scratch_bytes, h2b_stream_t stream);
/* culib.rs:579-592 ; ntt.cu:898-962 -- device outputs, input residency per input_on_device */
RustError _halo2_fft_many_to_device(uint32_t ntt_type, uint32_t num_many, uint32_t log_n, uint32_t extend_log_n,
                                    const FFITraitObject* input, const FFITraitObject* output,
                                    const void* omega_device, const FFITraitObject* divisor, bool input_on_device,
                                    void* scratch, uint64_t scratch_bytes, h2b_stream_t stream);
/* culib.rs:594 ; ntt.cu:792-800 -- always true */
bool _halo2_fft_many_check_memory(uint32_t ntt_type, uint32_t log_n, uint32_t extend_log_n);
/* culib.rs:596-601 ; ntt.cu:676-690 */
int32_t _halo2_get_fft_split_radix(uint32_t ntt_type, uint32_t log_n, uint32_t extend_log_n, uint64_t free_bytes);

/* ------------------------------------------------------------ twiddles --- */
/* culib.rs:428 declares `cuda_omega_lut(res, log_n)`, but the reference's
 * CUDA sources define no such symbol (nothing can call it); it has no
 * counterpart here either. */

/* culib.rs:430 ; polynomial/omega.cu:15-20 ; 0 when log_n >= 32 */
uint64_t _halo2_power_of_omega_workspace_size(uint32_t log_n);
/* culib.rs:432-441 ; polynomial/omega.cu:29-67 -- host omega in; host res = omega^pow and host
 * omega_lut[0..=log_n] = [1, omega, omega^2, omega^4, ...]; synchronises.  Code 1 when
 * log_n >= 32 or pow >= 2^log_n. */
RustError _halo2_power_of_omega(const FFITraitObject* res, const FFITraitObject* omega_lut,
                                const FFITraitObject* omega, uint32_t log_n, uint32_t pow, void* scratch,
                                uint64_t scratch_bytes, h2b_stream_t stream);
/* culib.rs:443 ; polynomial/omega.cu:72-75 */
uint64_t _halo2_generate_omega_powers_workspace_size(uint32_t log_n);
/* culib.rs:449-456 ; polynomial/omega.cu:77-94 -- device out[i] = omega^i, i < 2^log_n, from a
 * device omega; does not synchronise */
RustError _halo2_generate_omega_powers(void* d_omega_powers, const void* d_omega, uint32_t log_n, void* scratch,
                                       uint64_t scratch_bytes, h2b_stream_t stream);
/* culib.rs:458 ; polynomial/omega.cu:99-105 ; 0 outside [10, 42) */
uint64_t _halo2_generate_omega_lut_workspace_size(uint32_t log_n);
/* culib.rs:460-467 ; polynomial/omega.cu:107-150 -- host omega in; host table
 * [omega^i, i < 2^10] ++ [(omega^1024)^i, i < 2^(log_n-10)]; synchronises.  Code 1 outside
 * 10 <= log_n < 42. */
RustError _halo2_generate_omega_lut(const FFITraitObject* sparse_twiddle, const FFITraitObject* omega,
                                    uint32_t log_n, void* scratch, uint64_t scratch_bytes, h2b_stream_t stream);
/* culib.rs:469-475 ; polynomial/omega.cu:153-161 */
uint64_t _halo2_generate_omegadelta_workspace_size(uint32_t log_n, uint32_t omega_start, uint32_t omega_end,
                                                   uint32_t colunm_num, uint32_t colunm_offset);
/* culib.rs:477-490 ; polynomial/omega.cu:163-200 -- device res[i] = omega^row * delta^col for the
 * u32 pairs (col, row) = mapping[2 (omega_start + i) .. +1], i <= omega_end - omega_start; host
 * omega and delta; colunm_offset is unused (as in the reference kernel); does not synchronise. */
RustError _halo2_generate_omegadelta(void* res, const void* mapping, const void* omega, const void* delta,
                                     uint32_t log_n, uint32_t omega_start, uint32_t omega_end, uint32_t colunm_num,
                                     uint32_t colunm_offset, void* scratch, uint64_t scratch_bytes,
                                     h2b_stream_t stream);

/* ------------------------------------------------------------ quotient --- */

/* quotient.cu:334-345 -- rule decoding hook with no outputs (no Rust caller) */
void _halo2_quotient_decode(uint64_t* rules, uint64_t num_rules, uint64_t num_quotient, uint64_t rotation_scale,
                            uint64_t row_start, uint64_t row_end);

/* evaluation.rs:1435-1449 ; quotient.cu:190-222 */
uint64_t _halo2_evaluate_h_max_rows(const uint64_t* rules, uint64_t num_rules, uint64_t num_vp_rules,
                                    uint64_t num_quotient, uint64_t num_fixed, uint64_t num_instance,
                                    uint64_t num_advice, uint64_t num_challenges, uint64_t num_constants,
                                    uint64_t rotation_scale, uint64_t row_start, uint64_t row_end,
                                    uint64_t free_bytes);
/* evaluation.rs:1451-1464 ; quotient.cu:224-260 */
uint64_t _halo2_quotient_workspace_size(const uint64_t* rules, uint64_t num_rules, uint64_t num_vp_rules,
                                        uint64_t num_quotient, uint64_t num_fixed, uint64_t num_instance,
                                        uint64_t num_advice, uint64_t num_challenges, uint64_t num_constants,
                                        uint64_t rotation_scale, uint64_t row_start, uint64_t row_end);
/* evaluation.rs:1466-1490 ; quotient.cu:309-440 -- host columns and host output */
RustError _halo2_quotient(const FFITraitObject* fixed, uint64_t num_fixed, const FFITraitObject* instance,
                          uint64_t num_instance, const FFITraitObject* advices, uint64_t num_advice,
                          FFITraitObject challenges, uint64_t num_challenges, FFITraitObject constants,
                          uint64_t num_constants, FFITraitObject expr_constants, const uint64_t* rules,
                          uint64_t num_rules, const uint64_t* value_part_rules, uint64_t num_vp_rules,
                          FFITraitObject quotient_poly, uint64_t num_quotient, uint64_t rotation_scale,
                          uint64_t row_start, uint64_t row_end, void* scratch, uint64_t scratch_bytes,
                          h2b_stream_t stream);
/* evaluation.rs:1498-1522 ; quotient.cu:570-710 -- device column pointers, device output */
RustError _halo2_quotient_device_columns_device_out(
    const void* const* fixed_d_ptrs, uint64_t num_fixed, const void* const* instance_d_ptrs, uint64_t num_instance,
    const void* const* advice_d_ptrs, uint64_t num_advice, FFITraitObject challenges, uint64_t num_challenges,
    FFITraitObject constants, uint64_t num_constants, FFITraitObject expr_constants, const uint64_t* rules,
    uint64_t num_rules, const uint64_t* value_part_rules, uint64_t num_vp_rules, void* quotient_poly_device_ptr,
    uint64_t num_quotient, const void* prev_values_device_ptr, uint64_t rotation_scale, uint64_t row_start,
    uint64_t row_end, void* scratch, uint64_t scratch_bytes, h2b_stream_t stream);
/* evaluation.rs:1536-1559 ; quotient.cu:450-568 -- device column pointers, host output */
RustError _halo2_quotient_device_columns(const void* const* fixed_d_ptrs, uint64_t num_fixed,
                                         const void* const* instance_d_ptrs, uint64_t num_instance,
                                         const void* const* advice_d_ptrs, uint64_t num_advice,
                                         FFITraitObject challenges, uint64_t num_challenges,
                                         FFITraitObject constants, uint64_t num_constants,
                                         FFITraitObject expr_constants, const uint64_t* rules, uint64_t num_rules,
                                         const uint64_t* value_part_rules, uint64_t num_vp_rules,
                                         FFITraitObject quotient_poly, uint64_t num_quotient,
                                         uint64_t rotation_scale, uint64_t row_start, uint64_t row_end,
                                         void* scratch, uint64_t scratch_bytes, h2b_stream_t stream);
/* Resident quotient programs (no counterpart in the reference, which compiles and uploads its rule list,
 * constants and column table on every _halo2_quotient* call): h2b_quotient_program_build compiles the same rule
 * encoding once, binds it to its device columns (d_columns: host array of device pointers, fixed then instance
 * then advice) and uploads it into caller-owned device memory (h2b_quotient_program_size bytes; the call
 * synchronises `stream` once); h2b_quotient_program_run is then a kernel launch alone (no host copy, no
 * synchronisation), so it can run from many streams and inside a captured CUDA graph.  Output rows as
 * _halo2_quotient_device_columns_device_out. */
typedef struct h2b_quotient_program {
    uint32_t n_ops, n_vp, slots, reserved;
    uint64_t num_quotient;
    uint64_t off_vps, off_cols, off_consts, off_chal, off_y, bytes;
} h2b_quotient_program;
uint64_t h2b_quotient_program_size(uint64_t num_rules, uint64_t num_vp, uint64_t num_columns, uint64_t num_constants,
                                   uint64_t num_challenges);
RustError h2b_quotient_program_build(const uint64_t* rules, uint64_t num_rules, const uint64_t* value_part_rules,
                                     uint64_t num_vp, uint64_t num_fixed, uint64_t num_instance, uint64_t num_advice,
                                     const void* const* d_columns, const void* constants, uint64_t num_constants,
                                     const void* challenges, uint64_t num_challenges, const void* y,
                                     uint64_t num_quotient, uint64_t rotation_scale, void* d_program,
                                     uint64_t program_bytes, h2b_quotient_program* info, h2b_stream_t stream);
RustError h2b_quotient_program_run(const h2b_quotient_program* info, const void* d_program, void* d_out,
                                   const void* d_prev, uint64_t row_start, uint64_t row_end, h2b_stream_t stream);

/* Fused extended-part quotient (no counterpart in the reference: it replaces the
 * per-part sequence of evaluation.rs:1107-1417 -- _halo2_quotient_device_columns_device_out
 * for the gates, _halo2_quotient_permutation, and per lookup the product expression
 * through _halo2_quotient_device_columns_device_out into table_values followed by
 * _halo2_quotient_lookups -- with one kernel that evaluates all of it per row and
 * writes the accumulator once):
 *   out[(r - row_start) * out_stride + out_offset] = value(r) * scale   (scale optional)
 * value(r) equals the composition of those launchers with prev = 0: the gate value
 * parts in Horner order in y, then the permutation constraints (same arguments and
 * rotation rules as _halo2_quotient_permutation over the rows of this call), then for
 * each lookup its five constraints with table_values(r) = Horner(0, y, the product
 * expression's value parts) and rows r +- 1 taken mod num_quotient. With out_stride =
 * the number of extended parts, out_offset = the part and scale = 1 / t_evaluations[part]
 * the result is the part's slice of _halo2_extended_from_lagrange_vec_device followed by
 * _halo2_divide_by_vanishing_poly.
 * Columns, sigma, product and lookup cosets and l0 / l_last / l_active are device
 * pointers given in HOST arrays; y, beta, gamma, delta, delta_start, the coset shift,
 * omega, scale, constants and challenges are HOST 32-byte Montgomery values (the whole
 * program travels as the kernel's parameters: no device memory, no synchronisation,
 * capturable in a CUDA graph). Limits: 64 columns, 256 compiled ops, 64 value parts,
 * 192 constants, 16 challenges, 64 live intermediates, 8 permutation sets of at most
 * 32 columns, 8 lookups; beyond them it returns cudaErrorInvalidValue and the separate
 * entry points apply. */
typedef struct h2b_quotient_rules {
    const uint64_t* rules;            /* 2 words per rule, the reference encoding */
    uint64_t num_rules;
    const uint64_t* value_part_rules;
    uint64_t num_vp;
    const void* constants;            /* host, 32 bytes each */
    uint64_t num_constants;
    const void* challenges;           /* host, 32 bytes each */
    uint64_t num_challenges;
} h2b_quotient_rules;
typedef struct h2b_quotient_permutation_args {
    uint64_t n_sets, chunk_len, n_columns;
    const void* const* product_cosets;   /* n_sets device pointers */
    const void* const* sigma_cosets;     /* n_columns device pointers */
    const void* const* column_values;    /* n_columns device pointers, permutation column order */
    const void* beta;
    const void* gamma;
    const void* delta;
    const void* delta_start;
    const void* current_extended_omega;
    const void* omega;
    int32_t last_rotation, rot_scale, isize, reserved;
} h2b_quotient_permutation_args;
typedef struct h2b_quotient_lookup_args {
    h2b_quotient_rules product;          /* the (input + beta)(table + gamma) expression */
    const void* product_coset;
    const void* permuted_input_coset;
    const void* permuted_table_coset;
    const void* beta;
    const void* gamma;
} h2b_quotient_lookup_args;
RustError h2b_quotient_fused(const void* const* fixed, uint64_t num_fixed, const void* const* instance,
                             uint64_t num_instance, const void* const* advice, uint64_t num_advice,
                             const h2b_quotient_rules* gates, const void* y, const void* l0, const void* l_last,
                             const void* l_active_row, const h2b_quotient_permutation_args* perm /* nullable */,
                             const h2b_quotient_lookup_args* lookups, uint64_t num_lookups, uint64_t num_quotient,
                             uint64_t rotation_scale, uint64_t row_start, uint64_t row_end, void* out,
                             uint64_t out_stride, uint64_t out_offset, const void* scale /* nullable */,
                             h2b_stream_t stream);
/* register budget of the fused kernel: 3 (default), 4 or 5 blocks of 128 threads per SM; same results */
void h2b_quotient_fused_set_blocks(int blocks_per_sm);
int h2b_quotient_fused_get_blocks(void);
/* culib.rs:603-617 ; quotient_lookups.cu:16-53 -- all device pointers */
RustError _halo2_quotient_lookups(void* values, const void* table_values, const void* product_coset,
                                  const void* permuted_input_coset, const void* permuted_table_coset, const void* l0,
                                  const void* l_last, const void* l_active_row, const void* beta, const void* gamma,
                                  const void* y, uint64_t poly_length, h2b_stream_t stream);
/* culib.rs:622-650 ; permutation_quotient.cu:23-93 -- device buffers / pointer tables, host scalars */
RustError _halo2_quotient_permutation(void* values, const void* l0, const void* l_last, const void* l_active_row,
                                      const void* perm_prod_cosets, const void* perm_cosets, const void* column_values,
                                      const void* beta, const void* gamma, const void* y, const void* delta,
                                      const void* delta_start, const void* current_extended_omega, const void* omega,
                                      uint64_t n_sets, uint64_t chunk_len, uint64_t n_perm_cols, int32_t last_rotation,
                                      int32_t rot_scale, int32_t isize_, uint64_t poly_length, h2b_stream_t stream);

/* ------------------------------------------- additions of this library --- */
/* No counterpart in the reference.  Device-output, sync-free forms used by the
 * batched and served provers, plus tuning hooks. */

/* Same as _halo2_multiexp_device_scalars_device_bases but writes the 96-byte
 * result to d_out on `stream` without synchronising. */
RustError h2b_msm_device(const void* d_scalar, const void* d_bases, void* d_out, uint64_t length, void* scratch,
                         uint64_t scratch_bytes, h2b_stream_t stream);
/* Window bits (0 = automatic; 4..22 accepted, other values also mean automatic) and sorted entries per
 * accumulation chunk (0 = automatic). */
void h2b_msm_set_tuning(int window_bits, int chunk);
/* Form of the MSM bucket-accumulation kernel: 6 = lazy R' = 2^260 limbs of 52 bits on the FP64 pipe
 * (default; window-table MSMs use it too); 0 = lazy R = 2^261 limbs of 29 bits with one-step carries on the
 * integer multiply pipe (window-table MSMs use it for every choice but 6).  A library built with
 * H2B_EXPERIMENTS=1 also has the normalised R = 2^256 forms 1..5 (slower; A/B comparisons only).  A value
 * that is not built leaves the setting unchanged.  Same results; tuning only. */
void h2b_msm_set_accumulate_variant(int variant);
int h2b_msm_get_accumulate_variant(void);
/* Batch-affine pairing rounds before the XYZZ bucket accumulation (default 0; 1..3 only in a library built
 * with H2B_EXPERIMENTS=1, where they measured slower).  Same results; the MSM workspace-size queries depend on
 * it (set it before sizing scratch). */
void h2b_msm_set_pair_rounds(int rounds);
int h2b_msm_get_pair_rounds(void);

/* Precomputed window tables (no counterpart in the reference): an SRS kept resident with its window
 * multiples [2^(c w)] P_i, so an MSM over it reduces one bucket set and has no final doubling chain.
 * The table is opaque to callers: its points are stored as x * 2^261 mod p images, the form the
 * accumulation kernel reads, with the endomorphism images (beta x, y) of all slices after them.
 * h2b_msm_table_points: affine points in the table for n bases (0 if n is out of range). */
uint64_t h2b_msm_table_points(uint64_t n);
uint64_t h2b_msm_table_precompute_workspace_size(uint64_t n);
RustError h2b_msm_table_precompute(const void* d_bases, uint64_t n, void* d_table, void* scratch,
                                   uint64_t scratch_bytes, h2b_stream_t stream);
/* MSM of n <= table_n device scalars over a table built for table_n bases; 96-byte result at d_out (device). */
uint64_t h2b_msm_table_workspace_size(uint64_t n, uint64_t table_n);
RustError h2b_msm_device_table(const void* d_scalars, const void* d_table, uint64_t table_n, void* d_out, uint64_t n,
                               void* scratch, uint64_t scratch_bytes, h2b_stream_t stream);

/* Batch execution (no counterpart in the reference, which runs one launcher at a time on one stream).
 * h2b_exec_fork: `n` (1..32) internal non-blocking streams of the current device and calling thread, ordered
 * after `parent`; created on the first fork by that thread on that device and kept until exit (threads never
 * share them).  h2b_exec_join: `parent` waits for them; call it from the thread that forked. */
RustError h2b_exec_fork(h2b_stream_t parent, uint32_t n, h2b_stream_t* out_streams);
RustError h2b_exec_join(h2b_stream_t parent, uint32_t n);
/* Stream-ordered upload of `bytes` from host memory (pageable is staged before the call returns) without
 * waiting for the work already queued on `stream` (scalars and small tables between kernels). */
RustError h2b_upload(void* d_dst, const void* h_src, uint64_t bytes, h2b_stream_t stream);
/* Capture what is issued on `s` (and on streams forked from it) into a CUDA graph; replay it with
 * h2b_graph_launch.  Only calls without host copies or synchronisation can be captured. */
RustError h2b_graph_begin(h2b_stream_t s);
RustError h2b_graph_end(h2b_stream_t s, void** handle);
RustError h2b_graph_launch(void* handle, h2b_stream_t s);
void h2b_graph_destroy(void* handle);
/* `count` device-resident MSMs overlapped on `streams` forked streams (longest first onto the least-loaded
 * stream); each result is the 96-byte Jacobian image at d_out.  Scratch: h2b_msm_batch_workspace_size. */
typedef struct h2b_msm_job {
    const void* d_scalars;
    const void* d_bases;   /* plain bases, or a window table built for table_n bases */
    void* d_out;
    uint64_t n;
    uint64_t table_n;      /* 0: plain bases */
} h2b_msm_job;
uint64_t h2b_msm_batch_workspace_size(const h2b_msm_job* jobs, uint64_t count, uint32_t streams);
RustError h2b_msm_batch(const h2b_msm_job* jobs, uint64_t count, uint32_t streams, void* scratch,
                        uint64_t scratch_bytes, h2b_stream_t stream);
/* Up to 64 MSMs over ONE window table (every job names the same d_bases and table_n > 0; lengths may
 * differ, each <= table_n) run as one MSM: one counting sort with job j's entries in bucket set j, one
 * accumulation, one bucket reduction, one final kernel writing each job's 96-byte result to its d_out.
 * Same results as h2b_msm_device_table per job (no counterpart in the reference, which commits one
 * polynomial per _halo2_multiexp* call).  Scratch: h2b_msm_merged_workspace_size (0 if the jobs do not
 * qualify).  No host synchronisation; device outputs. */
uint64_t h2b_msm_merged_workspace_size(const h2b_msm_job* jobs, uint64_t count);
RustError h2b_msm_merged(const h2b_msm_job* jobs, uint64_t count, void* scratch, uint64_t scratch_bytes,
                         h2b_stream_t stream);
/* Batch inversion whose CTAs share a single inversion through scratch
 * (h2b_batch_invert_workspace_size bytes); same semantics as _halo2_batch_invert. */
uint64_t h2b_batch_invert_workspace_size(uint64_t length);
RustError h2b_batch_invert(void* d_data, uint32_t field_type, uint64_t length, void* scratch, uint64_t scratch_bytes,
                           h2b_stream_t stream);
/* Radix-2 stages per shared-memory NTT pass (1..11; radix-2 pass kernels take at most 10, radix-4 ones 11). */
void h2b_ntt_set_pass_stages(int stages);
int h2b_ntt_get_pass_stages(void);
/* NTT passes as radix-4 steps (1: a thread runs two stages on four elements in registers) or radix-2
 * stages (0).  Same results. */
void h2b_ntt_set_radix4(int on);
int h2b_ntt_get_radix4(void);
/* Per-size tuning table written by the autotuner (no counterpart in the reference, whose MSM window width
 * and NTT stage split are fixed formulas: halo2_proofs/cuda/src/multiexp.cu:260-300,
 * halo2_proofs/cuda/include/kernel/ntt_combine.h:90-94).  param 0 = MSM window bits (10..16; plain-base
 * MSMs only), 1 = MSM sorted entries per accumulation chunk (8..512; plain-base MSMs that run alone), 2 = NTT radix-2
 * stages per shared-memory pass (1..11; at most 10 with the radix-2 pass kernel), each for inputs of 2^log_n (floor of log2 for an MSM).  value 0 =
 * automatic.  Results never change, only times; MSM workspace sizes depend on entries 0 and 1, so set them
 * before sizing scratch.  h2b_tune_set returns 0, or -1 for an unknown param, log_n > 32 or a value out of
 * range (the table is then unchanged). */
int32_t h2b_tune_set(uint32_t param, uint32_t log_n, int32_t value);
int32_t h2b_tune_get(uint32_t param, uint32_t log_n);
void h2b_tune_clear(void);

/* ---------------------------------------- synthetic inputs (no reference counterpart) --- */

/* n Montgomery Fr from a seed: mix 0 uniform, mix 1 the witness-like mix of the k = 22 MSM
 * workload (50 % uniform, 30 % uniform below 2^64, 20 % in {0, 1}). */
RustError h2b_random_fr(void* d_out, uint64_t n, uint64_t seed, int mix, h2b_stream_t stream);
/* out[i] = x^i for i < n (d_x: one device Fr). */
RustError h2b_powers(void* d_out, uint64_t n, const void* d_x, h2b_stream_t stream);
/* out[i] = [s_i] G (affine, 64 B) for n device scalars, by fixed-base double-and-add over the
 * caller's device table of 2^j G, j < 256; with s_i = tau^i the synthetic KZG SRS
 * (unsafe_setup_with_s, halo2_proofs/src/poly/kzg/commitment.rs:132-200). */
RustError h2b_srs_from_powers(void* d_out, const void* d_scalars, uint64_t n, const void* d_table256,
                              h2b_stream_t stream);
/* out[0] = s0, out[1] = s1, out[i + 2] = out[i + 1] + out[i] (d_seeds: two device Fr): the
 * witness of a Fibonacci rotation gate. */
RustError h2b_fibonacci_fr(void* d_out, uint64_t n, const void* d_seeds, h2b_stream_t stream);
/* out[i] = table[idx[i]] for 32-byte elements (idx: n device int64); an index outside
 * [0, table_len) gives zero.  A witness column drawn from a table of values. */
RustError h2b_gather_fr(void* d_out, const void* d_table, uint64_t table_len, const int64_t* d_idx, uint64_t n,
                        h2b_stream_t stream);

/* ------------------------------------- measurement hooks (no reference counterpart) --- */

/* MSM window width the built-in plan takes for n plain bases. */
int h2b_msm_window_bits(uint64_t n);
/* Nonzero signed digits (= sorted bucket entries) of the plain MSM of n device scalars, as one
 * device uint64 at d_count. */
RustError h2b_msm_count_entries(const void* d_scalars, uint64_t n, void* d_count, h2b_stream_t stream);
/* Kernel launches this library has issued in the process. */
uint64_t h2b_launch_count(void);
/* CUDA-event timing of instrumented phases (id 0 MSM accumulation, 1 MSM total, 2 NTT passes,
 * 3 batch inversion, 4 quotient, 5 permute-sort): enable, then read the summed ms and count. */
void h2b_prof_enable(int on);
int h2b_prof_read(int id, double* total_ms, int* count);
/* Throughput probes: independent mad.lo / mad.hi chains, and four independent field products per
 * thread in registers (the product-rate reference of the rooflines); d_sink receives results. */
RustError h2b_probe_imad(int blocks, int threads, int iters, void* d_sink, h2b_stream_t stream);
RustError h2b_probe_modmul(int blocks, int threads, int iters, void* d_sink, h2b_stream_t stream);
/* out[i] = a[i] * b[i] with product implementation `impl` (tests: 0-2 Fr CIOS lo/hi, CIOS wide,
 * 29-bit; 3 Fr square; 4 Fq product; 5 Fq square; 6 Fr, 7 Fq with the FP64 form). */
RustError h2b_fr_mul_batch(int impl, const void* d_a, const void* d_b, void* d_out, uint64_t n,
                           h2b_stream_t stream);
/* MSM accumulation: prefetch into L2 the point this many sorted entries ahead (0..64, default 2;
 * 0 turns it off).  Same results. */
void h2b_msm_set_prefetch(int distance);
int h2b_msm_get_prefetch(void);

/* No counterpart in the reference.  Batch inversion with the semantics of
 * _halo2_batch_invert (in place, zeros stay zero, field_type 0 = Fr, 1 = Fq)
 * for callers that cannot allocate device memory: it keeps the scratch-free
 * call shape and uses a fixed 1.5 MiB array inside the library instead of a
 * workspace, so it allocates and frees nothing.  length <= 2^26 (larger is
 * an error).  All calls share that array: calls that overlap on the GPU
 * race, so serialise them on one stream.  The first call on each device
 * (and the first after its CUDA context is recreated) looks up the array's
 * address; make it before any stream capture. */
RustError h2b_batch_invert_noalloc(void* d_data, uint32_t field_type, uint64_t length, h2b_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* HALO2_GPU_H */
