// Root-of-unity tables (the reference's twiddle entry points,
// halo2_proofs/cuda/src/polynomial/omega.cu:15-200, bound at
// halo2_proofs/src/cuda/culib.rs:428-490 and wrapped by
// halo2_proofs/src/cuda/funcs/omega.rs):
//
//  * _halo2_power_of_omega: omega^pow and the log table
//    [1, omega, omega^2, omega^4, ..., omega^(2^(log_n-1))], both to host.
//  * _halo2_generate_omega_powers: omega^i for i < 2^log_n into a device
//    buffer (no synchronisation).
//  * _halo2_generate_omega_lut: the two-level table
//    [omega^i, i < 2^10] ++ [(omega^(2^10))^i, i < 2^(log_n-10)] to host
//    (DENSE_POWER_DEGREE = 10, halo2_proofs/src/arithmetic.rs).
//  * _halo2_generate_omegadelta: out[i] = omega^row * delta^col for the
//    (col, row) pairs mapping[start..=end] (u32 pairs), into a device buffer.
//
// Every table is built from a squaring chain lut[j] = x^(2^j) (one thread)
// and a coalesced power kernel: thread t of a block owning the index tile
// [b*T*K, (b+1)*T*K) starts at x^(b*T*K + t) (product of chain entries) and
// steps by x^T, so each warp stores 32 consecutive elements per step.
// Products are exact Montgomery products, so the tables are bit-identical to
// the reference's (whose kernels use a different multiplication order).
// Few product sites per kernel here: inline them (full product throughput).
#define H2B_INLINE_MUL 1
#include <algorithm>
#include <cstdio>
#include "abi.cuh"
#include "field.cuh"

namespace h2b {

namespace {
constexpr int PW_T = 256;
constexpr int PW_LOGT = 8;
constexpr int PW_K = 16;
constexpr uint32_t DENSE_DEGREE = 10;
}

// lut[j] = x^(2^j) for j < k; optionally lut0 gets 1 and the chain starts at
// index `shift` (the log-table layout of _halo2_power_of_omega).
static __global__ void k_square_chain(const Fr* __restrict__ x, Fr* __restrict__ lut, int k, int shift)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    if (shift) st(&lut[0], Fr::one());
    Fr cur = ld(x);
    for (int j = 0; j < k; j++) {
        st(&lut[j + shift], cur);
        cur = cur * cur;
    }
}

static __device__ __forceinline__ Fr pow_by_chain(const Fr* __restrict__ chain, uint64_t e)
{
    Fr r = Fr::one();
    for (int j = 0; e; j++, e >>= 1)
        if (e & 1) r = r * ldg(&chain[j]);
    return r;
}

// res = prod over set bits b of pow of loglut[b + 1] (loglut[0] = 1).
static __global__ void k_power_from_log_lut(const Fr* __restrict__ loglut, uint32_t pow, Fr* __restrict__ res)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    st(res, pow_by_chain(loglut + 1, pow));
}

// out[i] = x^i for i < n; chain[j] = x^(2^j) must cover j <= max(bits(n-1), PW_LOGT).
static __global__ void __launch_bounds__(PW_T) k_powers_tile(const Fr* __restrict__ chain, Fr* __restrict__ out,
                                                              uint64_t n)
{
    uint64_t i = blockIdx.x * (uint64_t)(PW_T * PW_K) + threadIdx.x;
    if (i >= n) return;
    Fr p = pow_by_chain(chain, i);
    const Fr step = ldg(&chain[PW_LOGT]);
#pragma unroll 1
    for (int j = 0; j < PW_K && i < n; j++, i += PW_T) {
        st(&out[i], p);
        p = p * step;
    }
}

// out[i] = low[row & 1023] * high[row >> 10] * delta[col] for
// (col, row) = mapping[2 (start + i)], mapping[2 (start + i) + 1], i <= end - start.
// Pairs outside the tables give zero (the reference reads out of bounds).
static __global__ void k_omegadelta(Fr* __restrict__ out, const uint32_t* __restrict__ mapping,
                                    const Fr* __restrict__ low, const Fr* __restrict__ high, uint64_t high_len,
                                    const Fr* __restrict__ delta, uint64_t delta_len, uint64_t start, uint64_t count)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint2 cr = __ldg((const uint2*)mapping + start + i);
        const uint64_t hi = cr.y >> DENSE_DEGREE;
        Fr r = Fr::zero();
        if (cr.x < delta_len && hi < high_len)
            r = ldg(&low[cr.y & ((1u << DENSE_DEGREE) - 1)]) * ldg(&high[hi]) * ldg(&delta[cr.x]);
        st(&out[i], r);
    }
}

static uint32_t bit_width(uint64_t x) { return x ? 64 - __builtin_clzll(x) : 0; }

// Chain length the power kernel needs for n outputs.
static uint32_t chain_len(uint64_t n) { return std::max<uint32_t>(bit_width(n ? n - 1 : 0), PW_LOGT + 1); }

static RustError launch_powers(const Fr* chain, Fr* out, uint64_t n, cudaStream_t st)
{
    if (n == 0) return ok();
    const uint64_t tile = (uint64_t)PW_T * PW_K;
    k_powers_tile<<<(unsigned)((n + tile - 1) / tile), PW_T, 0, st>>>(chain, out, n);
    H2B_LAUNCHED("k_powers_tile");
    return ok();
}

// ---- scratch layouts (shared by the size queries and the launchers) --------

struct PowerOfOmegaLayout {
    static void plan(ScratchPlan& p, uint32_t log_n)
    {
        p.add(32);                     // omega
        p.add(32ull * (log_n + 1));    // log table
        p.add(32);                     // result
    }
};

static uint64_t lut_len(uint32_t log_n) { return (1ull << DENSE_DEGREE) + (1ull << (log_n - DENSE_DEGREE)); }

static bool lut_log_ok(uint32_t log_n) { return log_n >= DENSE_DEGREE && log_n < DENSE_DEGREE + 32; }

// chain of omega long enough for both table halves: the high half uses
// chain + 10 with its own bound.
static uint32_t lut_chain_len(uint32_t log_n)
{
    return std::max<uint32_t>(chain_len(1ull << DENSE_DEGREE), DENSE_DEGREE + chain_len(1ull << (log_n - DENSE_DEGREE)));
}

static uint32_t delta_log(uint32_t colnum)
{
    uint32_t l = 0;
    for (uint64_t c = 1; c < colnum; c <<= 1) l++;
    return l;
}

} // namespace h2b

using namespace h2b;

// ---------------------------------------------------------------------------
// omega.cu:15-67
extern "C" uint64_t _halo2_power_of_omega_workspace_size(uint32_t log_n)
{
    if (log_n >= 32) return 0;
    ScratchPlan p;
    PowerOfOmegaLayout::plan(p, log_n);
    return p.used;
}

extern "C" RustError _halo2_power_of_omega(const FFITraitObject* res, const FFITraitObject* omega_lut,
                                           const FFITraitObject* omega, uint32_t log_n, uint32_t pow, void* scratch,
                                           uint64_t scratch_bytes, cudaStream_t stream)
{
    if (log_n >= 32 || bit_width(pow) > log_n)
        return err((int)cudaErrorInvalidValue, "_halo2_power_of_omega: pow must be < (1 << log_n) and log_n < 32");
    ScratchArena a(scratch, scratch_bytes);
    Fr* d_omega = a.take_n<Fr>(1);
    Fr* d_lut = a.take_n<Fr>(log_n + 1);
    Fr* d_res = a.take_n<Fr>(1);
    if (!a.good()) return scratch_too_small("_halo2_power_of_omega", scratch_bytes,
                                            _halo2_power_of_omega_workspace_size(log_n));
    H2B_CUDA(cudaMemcpyAsync(d_omega, omega->ptr, 32, cudaMemcpyHostToDevice, stream));
    k_square_chain<<<1, 32, 0, stream>>>(d_omega, d_lut, (int)log_n, 1);
    H2B_LAUNCHED("k_square_chain");
    k_power_from_log_lut<<<1, 32, 0, stream>>>(d_lut, pow, d_res);
    H2B_LAUNCHED("k_power_from_log_lut");
    H2B_CUDA(cudaMemcpyAsync(omega_lut->ptr, d_lut, 32ull * (log_n + 1), cudaMemcpyDeviceToHost, stream));
    H2B_CUDA(cudaMemcpyAsync(res->ptr, d_res, 32, cudaMemcpyDeviceToHost, stream));
    H2B_CUDA(cudaStreamSynchronize(stream));
    return ok();
}

// omega.cu:72-94 -- device output, device omega, no synchronisation
extern "C" uint64_t _halo2_generate_omega_powers_workspace_size(uint32_t log_n)
{
    if (log_n >= 48) return 0;
    ScratchPlan p;
    p.add(32ull * chain_len(1ull << log_n));
    return p.used;
}

extern "C" RustError _halo2_generate_omega_powers(void* d_omega_powers, const void* d_omega, uint32_t log_n,
                                                  void* scratch, uint64_t scratch_bytes, cudaStream_t stream)
{
    if (log_n >= 48) return err((int)cudaErrorInvalidValue, "_halo2_generate_omega_powers: log_n must be < 48");
    const uint64_t n = 1ull << log_n;
    const uint32_t k = chain_len(n);
    ScratchArena a(scratch, scratch_bytes);
    Fr* chain = a.take_n<Fr>(k);
    if (!a.good()) return scratch_too_small("_halo2_generate_omega_powers", scratch_bytes,
                                            _halo2_generate_omega_powers_workspace_size(log_n));
    k_square_chain<<<1, 32, 0, stream>>>((const Fr*)d_omega, chain, (int)k, 0);
    H2B_LAUNCHED("k_square_chain");
    return launch_powers(chain, (Fr*)d_omega_powers, n, stream);
}

// omega.cu:99-150 -- host output, host omega, synchronises
extern "C" uint64_t _halo2_generate_omega_lut_workspace_size(uint32_t log_n)
{
    if (!lut_log_ok(log_n)) return 0;
    ScratchPlan p;
    p.add(32);                           // omega
    p.add(32ull * lut_chain_len(log_n));  // chain
    p.add(32ull * lut_len(log_n));        // table
    return p.used;
}

extern "C" RustError _halo2_generate_omega_lut(const FFITraitObject* omega_lut, const FFITraitObject* omega,
                                               uint32_t log_n, void* scratch, uint64_t scratch_bytes,
                                               cudaStream_t stream)
{
    if (!lut_log_ok(log_n))
        return err((int)cudaErrorInvalidValue, "_halo2_generate_omega_lut: log_n must be in [10, 42)");
    ScratchArena a(scratch, scratch_bytes);
    Fr* d_omega = a.take_n<Fr>(1);
    const uint32_t k = lut_chain_len(log_n);
    Fr* chain = a.take_n<Fr>(k);
    Fr* table = a.take_n<Fr>(lut_len(log_n));
    if (!a.good()) return scratch_too_small("_halo2_generate_omega_lut", scratch_bytes,
                                            _halo2_generate_omega_lut_workspace_size(log_n));
    H2B_CUDA(cudaMemcpyAsync(d_omega, omega->ptr, 32, cudaMemcpyHostToDevice, stream));
    k_square_chain<<<1, 32, 0, stream>>>(d_omega, chain, (int)k, 0);
    H2B_LAUNCHED("k_square_chain");
    H2B_TRY(launch_powers(chain, table, 1ull << DENSE_DEGREE, stream));
    H2B_TRY(launch_powers(chain + DENSE_DEGREE, table + (1ull << DENSE_DEGREE), 1ull << (log_n - DENSE_DEGREE), stream));
    H2B_CUDA(cudaMemcpyAsync(omega_lut->ptr, table, 32ull * lut_len(log_n), cudaMemcpyDeviceToHost, stream));
    H2B_CUDA(cudaStreamSynchronize(stream));
    return ok();
}

// omega.cu:153-200 -- device output and mapping, host omega and delta, no
// synchronisation.  colunm_offset is accepted and unused, as in the reference
// kernel (kernel/omega.h cukernel_generate_omegadelta).
static void omegadelta_plan(ScratchPlan& p, uint32_t log_n, uint32_t colnum)
{
    const uint32_t dl = delta_log(colnum);
    p.add(64);                                   // omega, delta
    p.add(32ull * lut_chain_len(log_n));          // omega chain
    p.add(32ull * chain_len(1ull << dl));         // delta chain
    p.add(32ull * lut_len(log_n));                // omega table
    p.add(32ull << dl);                           // delta table
}

extern "C" uint64_t _halo2_generate_omegadelta_workspace_size(uint32_t log_n, uint32_t omega_start,
                                                              uint32_t omega_end, uint32_t colunm_num,
                                                              uint32_t colunm_offset)
{
    (void)omega_start; (void)omega_end; (void)colunm_offset;
    if (!lut_log_ok(log_n)) return 0;
    ScratchPlan p;
    omegadelta_plan(p, log_n, colunm_num);
    return p.used;
}

extern "C" RustError _halo2_generate_omegadelta(void* omegadelta, const void* mapping, const void* omega_host,
                                                const void* delta_host, uint32_t log_n, uint32_t omega_start,
                                                uint32_t omega_end, uint32_t colunm_num, uint32_t colunm_offset,
                                                void* scratch, uint64_t scratch_bytes, cudaStream_t stream)
{
    (void)colunm_offset;
    if (!lut_log_ok(log_n))
        return err((int)cudaErrorInvalidValue, "_halo2_generate_omegadelta: log_n must be in [10, 42)");
    if (omega_end < omega_start)
        return err((int)cudaErrorInvalidValue, "_halo2_generate_omegadelta: omega_end < omega_start");
    const uint32_t dl = delta_log(colunm_num);
    const uint32_t kw = lut_chain_len(log_n), kd = chain_len(1ull << dl);
    ScratchArena a(scratch, scratch_bytes);
    Fr* d_wd = a.take_n<Fr>(2);
    Fr* chain_w = a.take_n<Fr>(kw);
    Fr* chain_d = a.take_n<Fr>(kd);
    Fr* table_w = a.take_n<Fr>(lut_len(log_n));
    Fr* table_d = a.take_n<Fr>(1ull << dl);
    if (!a.good()) {
        ScratchPlan p;
        omegadelta_plan(p, log_n, colunm_num);
        return scratch_too_small("_halo2_generate_omegadelta", scratch_bytes, p.used);
    }
    H2B_CUDA(cudaMemcpyAsync(d_wd, omega_host, 32, cudaMemcpyHostToDevice, stream));
    H2B_CUDA(cudaMemcpyAsync(d_wd + 1, delta_host, 32, cudaMemcpyHostToDevice, stream));
    k_square_chain<<<1, 32, 0, stream>>>(d_wd, chain_w, (int)kw, 0);
    H2B_LAUNCHED("k_square_chain");
    k_square_chain<<<1, 32, 0, stream>>>(d_wd + 1, chain_d, (int)kd, 0);
    H2B_LAUNCHED("k_square_chain");
    H2B_TRY(launch_powers(chain_w, table_w, 1ull << DENSE_DEGREE, stream));
    const uint64_t high_len = 1ull << (log_n - DENSE_DEGREE);
    H2B_TRY(launch_powers(chain_w + DENSE_DEGREE, table_w + (1ull << DENSE_DEGREE), high_len, stream));
    H2B_TRY(launch_powers(chain_d, table_d, 1ull << dl, stream));
    const uint64_t count = (uint64_t)omega_end - omega_start + 1;
    k_omegadelta<<<grid_for(count, 256), 256, 0, stream>>>((Fr*)omegadelta, (const uint32_t*)mapping, table_w,
                                                          table_w + (1ull << DENSE_DEGREE), high_len, table_d,
                                                          1ull << dl, omega_start, count);
    H2B_LAUNCHED("k_omegadelta");
    return ok();
}
