// Synthetic-input generators that run on the device (setup utilities, not
// part of the reference ABI):
//  * h2b_random_fr: n seeded Fr elements (Montgomery form).  Element i draws
//    512 bits from a SplitMix64 stream keyed by (seed, i) and reduces them as
//    d0 * R^2 + d1 * R^3 -- the wide-reduction shape halo2curves' Fr::random
//    uses.  `mix` = 1 gives the witness-like mix of the k=22 MSM workload:
//    50% uniform, 30% uniform below 2^64, 20% uniform in {0, 1}.
//  * h2b_powers: out[i] = x^i.
//  * h2b_fibonacci_fr: out[0] = s0, out[1] = s1, out[i + 2] = out[i + 1] + out[i]
//    (the witness of a Fibonacci rotation gate).  out[i] = s0 F(i-1) + s1 F(i)
//    with F the Fibonacci numbers mod r, so each thread reaches its chunk
//    start by fast doubling (F(2m) = F(m)(2F(m+1) - F(m)),
//    F(2m+1) = F(m)^2 + F(m+1)^2) and then steps the recurrence.
//  * h2b_gather_fr: out[i] = table[idx[i]] for 32-byte field elements (a
//    witness column drawn from a table of values); an index outside the
//    table gives zero.
//  * h2b_srs_from_powers: out[i] = [s_i] G as affine points for Montgomery
//    scalars s_i, by fixed-base double-and-add over a caller-supplied table
//    of affine 2^j G (j < 256), then one inversion per point.  With
//    s_i = tau^i this is the synthetic KZG SRS of unsafe_setup_with_s
//    (halo2_proofs/src/poly/kzg/commitment.rs:132-200).
#include "abi.cuh"
#include "curve.cuh"

namespace h2b {

__device__ __forceinline__ uint64_t splitmix64(uint64_t& s)
{
    uint64_t z = (s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

__global__ void k_random_fr(Fr* __restrict__ out, uint64_t n, uint64_t seed, int mix)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t s = seed * 0xd1342543de82ef95ull + i * 0x2545f4914f6cdd1dull + 0x632be59bd9b4e019ull;
        uint64_t w[8];
        for (int k = 0; k < 8; k++) w[k] = splitmix64(s);
        Fr r;
        int cls = 0;
        if (mix == 1) {
            uint64_t u = splitmix64(s) % 10;  // 0-4 uniform, 5-7 small, 8-9 bit
            cls = u < 5 ? 0 : (u < 8 ? 1 : 2);
        }
        if (cls == 0) {
            Fr d0, d1;
            for (int k = 0; k < 4; k++) {
                d0.v[2 * k] = (uint32_t)w[k]; d0.v[2 * k + 1] = (uint32_t)(w[k] >> 32);
                d1.v[2 * k] = (uint32_t)w[4 + k]; d1.v[2 * k + 1] = (uint32_t)(w[4 + k] >> 32);
            }
            Fr r2 = Fr::r2();
            Fr r3 = r2 * r2;
            r = d0 * r2 + d1 * r3;
        } else {
            Fr c = Fr::zero();
            if (cls == 1) { c.v[0] = (uint32_t)w[0]; c.v[1] = (uint32_t)(w[0] >> 32); }
            else { c.v[0] = (uint32_t)(w[0] & 1u); }
            r = to_mont(c);
        }
        st(&out[i], r);
    }
}

constexpr int POW_CHUNK = 16;
__global__ void k_powers(Fr* __restrict__ out, uint64_t n, const Fr* __restrict__ px)
{
    const Fr x = ld(px);
    uint64_t nthreads = (n + POW_CHUNK - 1) / POW_CHUNK;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < nthreads;
         t += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t i0 = t * POW_CHUNK;
        Fr p = Fr::one(), b = x;
        for (uint64_t e = i0; e; e >>= 1) {
            if (e & 1) p = p * b;
            b = b * b;
        }
        for (int j = 0; j < POW_CHUNK && i0 + j < n; j++) {
            st(&out[i0 + j], p);
            p = p * x;
        }
    }
}

constexpr int FIB_CHUNK = 64;
__global__ void k_fibonacci(Fr* __restrict__ out, uint64_t n, const Fr* __restrict__ seeds)
{
    const Fr s0 = ld(&seeds[0]), s1 = ld(&seeds[1]);
    uint64_t nthreads = (n + FIB_CHUNK - 1) / FIB_CHUNK;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < nthreads;
         t += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t i0 = t * FIB_CHUNK;
        Fr a = Fr::zero(), b = Fr::one();          // (F(m), F(m + 1)) for m = the bits of i0 seen so far
        for (int bit = 63; bit >= 0; bit--) {
            if ((i0 >> bit) == 0) continue;
            Fr c = a * (b + b - a);
            Fr d = a * a + b * b;
            if ((i0 >> bit) & 1) { a = d; b = c + d; } else { a = c; b = d; }
        }
        Fr cur = s0 * (b - a) + s1 * a;            // out[i0] = s0 F(i0 - 1) + s1 F(i0)
        Fr nxt = s0 * a + s1 * b;                  // out[i0 + 1]
        for (int j = 0; j < FIB_CHUNK && i0 + j < n; j++) {
            st(&out[i0 + j], cur);
            Fr sum = cur + nxt;
            cur = nxt;
            nxt = sum;
        }
    }
}

__global__ void __launch_bounds__(128) k_srs(G1Affine* __restrict__ out, const Fr* __restrict__ scalars, uint64_t n,
                                             const G1Affine* __restrict__ table)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        Fr s = from_mont(ld(&scalars[i]));
        G1Xyzz acc = xyzz_inf();
        for (int j = 0; j < 256; j++) {
            if ((s.v[j >> 5] >> (j & 31)) & 1u) xyzz_madd(acc, ld_affine(&table[j]));
        }
        G1Affine a;
        if (is_inf(acc)) {
            a.x = Fq::zero(); a.y = Fq::zero();
        } else {
            G1Jac jj = xyzz_to_jac_affine(acc);
            a.x = jj.X; a.y = jj.Y;
        }
        st(&out[i].x, a.x);
        st(&out[i].y, a.y);
    }
}

} // namespace h2b

using namespace h2b;

extern "C" RustError h2b_random_fr(void* d_out, uint64_t n, uint64_t seed, int mix, cudaStream_t stream)
{
    if (n == 0) return ok();
    k_random_fr<<<grid_for(n, 256, 148u * 16u), 256, 0, stream>>>((Fr*)d_out, n, seed, mix);
    H2B_LAUNCHED("k_random_fr");
    return ok();
}

extern "C" RustError h2b_powers(void* d_out, uint64_t n, const void* d_x, cudaStream_t stream)
{
    if (n == 0) return ok();
    uint64_t nthreads = (n + POW_CHUNK - 1) / POW_CHUNK;
    k_powers<<<grid_for(nthreads, 256, 148u * 16u), 256, 0, stream>>>((Fr*)d_out, n, (const Fr*)d_x);
    H2B_LAUNCHED("k_powers");
    return ok();
}

extern "C" RustError h2b_fibonacci_fr(void* d_out, uint64_t n, const void* d_seeds, cudaStream_t stream)
{
    if (n == 0) return ok();
    uint64_t nthreads = (n + FIB_CHUNK - 1) / FIB_CHUNK;
    k_fibonacci<<<grid_for(nthreads, 128, 148u * 16u), 128, 0, stream>>>((Fr*)d_out, n, (const Fr*)d_seeds);
    H2B_LAUNCHED("k_fibonacci");
    return ok();
}

// One element per thread, two 16-byte loads and stores: HBM-bound.
__global__ void k_gather_fr(uint4* __restrict__ out, const uint4* __restrict__ table, uint64_t table_len,
                            const int64_t* __restrict__ idx, uint64_t n)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const int64_t j = idx[i];
        uint4 lo = make_uint4(0u, 0u, 0u, 0u), hi = lo;
        if (j >= 0 && (uint64_t)j < table_len) {
            lo = __ldg(&table[2 * j]);
            hi = __ldg(&table[2 * j + 1]);
        }
        out[2 * i] = lo;
        out[2 * i + 1] = hi;
    }
}

extern "C" RustError h2b_gather_fr(void* d_out, const void* d_table, uint64_t table_len, const int64_t* d_idx,
                                   uint64_t n, cudaStream_t stream)
{
    if (n == 0) return ok();
    if (!d_out || !d_idx || (table_len && !d_table))
        return err(cudaErrorInvalidValue, "h2b_gather_fr: null pointer");
    k_gather_fr<<<grid_for(n, 256, 148u * 16u), 256, 0, stream>>>((uint4*)d_out, (const uint4*)d_table, table_len,
                                                                  d_idx, n);
    H2B_LAUNCHED("k_gather_fr");
    return ok();
}

extern "C" RustError h2b_srs_from_powers(void* d_out, const void* d_scalars, uint64_t n, const void* d_table256,
                                         cudaStream_t stream)
{
    if (n == 0) return ok();
    k_srs<<<grid_for(n, 128, 148u * 32u), 128, 0, stream>>>((G1Affine*)d_out, (const Fr*)d_scalars, n,
                                                           (const G1Affine*)d_table256);
    H2B_LAUNCHED("k_srs");
    return ok();
}
