// Element-wise polynomial entry points around the quotient
// (halo2_proofs/cuda/src/polynomial/polynomial.cu:247-455, declared at
// halo2_proofs/src/cuda/culib.rs:276-399):
//   extended_from_lagrange_vec : out[i*P + p] = part_p[i]           (domain.rs:173-220)
//   divide_by_vanishing_poly   : a_i *= t[i mod t_len]               (domain.rs:702-726)
//   distribute_powers_zeta     : a_i *= c[(i mod (L+1)) - 1], i mod (L+1) != 0
//   elementwise multiply, fill with one, multiply-add, short subtractions.
// All are HBM-bound streaming kernels: one 32-byte load/store per operand,
// grid sized to a few waves of the 148 SMs.
// Few product sites per kernel here: inline them (full product throughput).
#define H2B_INLINE_MUL 1
#include "abi.cuh"
#include "field.cuh"

namespace h2b {

constexpr unsigned EW_THREADS = 256;
constexpr unsigned EW_CAP = 148u * 8u;

#define H2B_GRID_STRIDE(i, n) \
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < (n); i += (uint64_t)gridDim.x * blockDim.x)

__global__ void k_extended_from_parts(Fr* __restrict__ out, const Fr* const* __restrict__ parts, uint32_t P, uint64_t n)
{
    // each thread writes one contiguous output element; reads are strided per part
    uint64_t total = n * P;
    H2B_GRID_STRIDE(j, total)
    {
        uint64_t i = j / P;
        uint32_t p = (uint32_t)(j - i * P);
        st(&out[j], ldg(&parts[p][i]));
    }
}

__global__ void k_divide_by_vanishing(Fr* __restrict__ a, const Fr* __restrict__ t, uint32_t tl, uint64_t n)
{
    H2B_GRID_STRIDE(i, n) { st(&a[i], ld(&a[i]) * ldg(&t[i % tl])); }
}

__global__ void k_distribute_powers(Fr* __restrict__ a, const Fr* __restrict__ c, uint32_t L, uint64_t n)
{
    const uint32_t mod = L + 1;
    H2B_GRID_STRIDE(i, n)
    {
        uint32_t r = (uint32_t)(i % mod);
        if (r != 0) st(&a[i], ld(&a[i]) * ldg(&c[r - 1]));
    }
}

__global__ void k_mul(Fr* out, const Fr* a, const Fr* b, uint64_t n)
{
    H2B_GRID_STRIDE(i, n) { st(&out[i], ld(&a[i]) * ld(&b[i])); }
}

__global__ void k_fill_one(Fr* __restrict__ out, uint64_t n)
{
    H2B_GRID_STRIDE(i, n) { st(&out[i], Fr::one()); }
}

__global__ void k_mul_add(Fr* __restrict__ acc, const Fr* __restrict__ in, const Fr* __restrict__ s, uint64_t n)
{
    const Fr k = ld(s);
    H2B_GRID_STRIDE(i, n) { st(&acc[i], ld(&acc[i]) + ld(&in[i]) * k); }
}

__global__ void k_sub_short(Fr* __restrict__ acc, const Fr* __restrict__ sh, uint64_t n)
{
    H2B_GRID_STRIDE(i, n) { st(&acc[i], ld(&acc[i]) - ld(&sh[i])); }
}

__global__ void k_sub_short_oop(Fr* __restrict__ out, const Fr* __restrict__ lg, const Fr* __restrict__ sh,
                                uint64_t short_len, uint64_t long_len)
{
    H2B_GRID_STRIDE(i, long_len)
    {
        Fr a = ld(&lg[i]);
        st(&out[i], i < short_len ? a - ld(&sh[i]) : a);
    }
}

__global__ void k_sub_scalar_at_zero(Fr* __restrict__ buf, const Fr* __restrict__ s)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) st(&buf[0], ld(&buf[0]) - ld(s));
}

} // namespace h2b

using namespace h2b;

extern "C" RustError _halo2_extended_from_lagrange_vec_device(void* d_out, const void* d_parts, uint32_t num_parts,
                                                              uint64_t n, cudaStream_t stream)
{
    if (n == 0 || num_parts == 0) return ok();
    k_extended_from_parts<<<grid_for(n * num_parts, EW_THREADS, EW_CAP), EW_THREADS, 0, stream>>>(
        (Fr*)d_out, (const Fr* const*)d_parts, num_parts, n);
    H2B_LAUNCHED("k_extended_from_parts");
    return ok();
}

extern "C" RustError _halo2_divide_by_vanishing_poly(void* d_poly, const void* d_t_evals, uint32_t t_len, uint64_t n,
                                                     cudaStream_t stream)
{
    if (n == 0) return ok();
    if (t_len == 0) return err(cudaErrorInvalidValue, "_halo2_divide_by_vanishing_poly: t_len must be >= 1");
    k_divide_by_vanishing<<<grid_for(n, EW_THREADS, EW_CAP), EW_THREADS, 0, stream>>>((Fr*)d_poly,
                                                                                      (const Fr*)d_t_evals, t_len, n);
    H2B_LAUNCHED("k_divide_by_vanishing");
    return ok();
}

extern "C" RustError _halo2_distribute_powers_zeta(void* d_a, const void* d_coset_powers, uint32_t coset_powers_len,
                                                   uint64_t n, cudaStream_t stream)
{
    if (n == 0 || coset_powers_len == 0) return ok();
    k_distribute_powers<<<grid_for(n, EW_THREADS, EW_CAP), EW_THREADS, 0, stream>>>(
        (Fr*)d_a, (const Fr*)d_coset_powers, coset_powers_len, n);
    H2B_LAUNCHED("k_distribute_powers");
    return ok();
}

extern "C" RustError _halo2_poly_elementwise_multiply(void* d_out, const void* d_a, const void* d_b, uint64_t length,
                                                      cudaStream_t stream)
{
    if (length == 0) return ok();
    k_mul<<<grid_for(length, EW_THREADS, EW_CAP), EW_THREADS, 0, stream>>>((Fr*)d_out, (const Fr*)d_a,
                                                                          (const Fr*)d_b, length);
    H2B_LAUNCHED("k_mul");
    return ok();
}

extern "C" RustError _halo2_poly_fill_one(void* d_out, uint64_t length, cudaStream_t stream)
{
    if (length == 0) return ok();
    k_fill_one<<<grid_for(length, EW_THREADS, EW_CAP), EW_THREADS, 0, stream>>>((Fr*)d_out, length);
    H2B_LAUNCHED("k_fill_one");
    return ok();
}

extern "C" RustError _halo2_poly_multiply_add(void* d_poly_acc, const void* d_poly_in, const void* d_scalar,
                                              uint64_t poly_length, cudaStream_t stream)
{
    if (poly_length == 0) return ok();
    k_mul_add<<<grid_for(poly_length, EW_THREADS, EW_CAP), EW_THREADS, 0, stream>>>(
        (Fr*)d_poly_acc, (const Fr*)d_poly_in, (const Fr*)d_scalar, poly_length);
    H2B_LAUNCHED("k_mul_add");
    return ok();
}

extern "C" RustError _halo2_poly_sub_short_inplace(void* d_acc, const void* d_short, uint64_t short_len,
                                                   cudaStream_t stream)
{
    if (short_len == 0) return ok();
    k_sub_short<<<grid_for(short_len, EW_THREADS, EW_CAP), EW_THREADS, 0, stream>>>((Fr*)d_acc,
                                                                                    (const Fr*)d_short, short_len);
    H2B_LAUNCHED("k_sub_short");
    return ok();
}

extern "C" RustError _halo2_poly_sub_short_out_of_place(void* d_out, const void* d_long, const void* d_short,
                                                        uint64_t short_len, uint64_t long_len, cudaStream_t stream)
{
    if (long_len == 0) return ok();
    k_sub_short_oop<<<grid_for(long_len, EW_THREADS, EW_CAP), EW_THREADS, 0, stream>>>(
        (Fr*)d_out, (const Fr*)d_long, (const Fr*)d_short, short_len, long_len);
    H2B_LAUNCHED("k_sub_short_oop");
    return ok();
}

extern "C" RustError _halo2_poly_sub_scalar_at_zero(void* d_buf, const void* d_scalar, cudaStream_t stream)
{
    k_sub_scalar_at_zero<<<1, 32, 0, stream>>>((Fr*)d_buf, (const Fr*)d_scalar);
    H2B_LAUNCHED("k_sub_scalar_at_zero");
    return ok();
}
