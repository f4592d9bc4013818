// Event-based kernel timing hook and pipe-throughput probes.
//
//  * h2b_prof_enable / h2b_prof_read: see prof.cuh.  Events come from a pool
//    created on first use; nothing here allocates device memory.
//  * h2b_probe_imad: independent mad.lo / mad.hi chains at full occupancy,
//    giving the measured 32-bit integer multiply-add throughput that bounds
//    every Montgomery-arithmetic kernel in this library.
//  * h2b_probe_modmul: four independent Montgomery products per thread per
//    iteration, the achievable Fr multiplication rate of field.cuh.
#include <mutex>
#include <vector>
#include "abi.cuh"
#include "field.cuh"
#include "prof.cuh"

// H2B_EXPERIMENTS=1 also builds the product-form probes used for A/B
// comparisons (h2b_probe_imad_form, h2b_probe_modmul_impl).
#ifndef H2B_EXPERIMENTS
#define H2B_EXPERIMENTS 0
#endif

namespace h2b {

namespace {
struct Pair {
    cudaEvent_t a, b;
};
std::mutex g_mu;
bool g_on = false;
std::vector<Pair> g_pool;
std::vector<Pair> g_used[PROF_IDS];
Pair g_open[PROF_IDS];
bool g_is_open[PROF_IDS];

Pair take_pair()
{
    if (!g_pool.empty()) {
        Pair p = g_pool.back();
        g_pool.pop_back();
        return p;
    }
    Pair p;
    cudaEventCreate(&p.a);
    cudaEventCreate(&p.b);
    return p;
}
} // namespace

bool prof_on() { return g_on; }

void prof_begin(int id, cudaStream_t st)
{
    if (!g_on || id < 0 || id >= PROF_IDS) return;
    std::lock_guard<std::mutex> lk(g_mu);
    Pair p = take_pair();
    cudaEventRecord(p.a, st);
    g_open[id] = p;
    g_is_open[id] = true;
}

void prof_end(int id, cudaStream_t st)
{
    if (!g_on || id < 0 || id >= PROF_IDS) return;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_is_open[id]) return;
    cudaEventRecord(g_open[id].b, st);
    g_used[id].push_back(g_open[id]);
    g_is_open[id] = false;
}

// 16 independent 32-bit IMADs per iteration per thread (8 lo, 8 hi).
__global__ void k_probe_imad(uint32_t* sink, int iters, uint32_t seed)
{
    uint32_t a[8];
    for (int j = 0; j < 8; j++) a[j] = seed * (threadIdx.x + 1) + j * 0x9e3779b9u;
    const uint32_t m = seed | 1u;
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int j = 0; j < 8; j++) {
            asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a[j]) : "r"(m), "r"(a[(j + 1) & 7]));
            asm volatile("mad.hi.u32 %0, %0, %1, %2;" : "+r"(a[j]) : "r"(m), "r"(a[(j + 3) & 7]));
        }
    }
    uint32_t x = 0;
    for (int j = 0; j < 8; j++) x ^= a[j];
    if (x == 0x12345678u) sink[blockIdx.x] = x;
}

// Single-form throughput: mode 0 = mad.lo.u32, 1 = mad.hi.u32, 2 = mad.wide.u32
// (16 independent instructions per iteration per thread).
#if H2B_EXPERIMENTS
__global__ void k_probe_imad_form(uint32_t* sink, int iters, uint32_t seed, int mode)
{
    uint32_t a[16];
    for (int j = 0; j < 16; j++) a[j] = seed * (threadIdx.x + 1) + j * 0x9e3779b9u;
    const uint32_t m = seed | 1u;
    if (mode == 0) {
        for (int it = 0; it < iters; it++) {
#pragma unroll
            for (int j = 0; j < 16; j++)
                asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a[j]) : "r"(m), "r"(a[(j + 5) & 15]));
        }
    } else if (mode == 1) {
        for (int it = 0; it < iters; it++) {
#pragma unroll
            for (int j = 0; j < 16; j++)
                asm volatile("mad.hi.u32 %0, %0, %1, %2;" : "+r"(a[j]) : "r"(m), "r"(a[(j + 5) & 15]));
        }
    } else {
        uint64_t w[8];
        for (int j = 0; j < 8; j++) w[j] = ((uint64_t)a[j] << 32) | a[j + 8];
        for (int it = 0; it < iters; it++) {
#pragma unroll
            for (int j = 0; j < 8; j++) {
                uint32_t lo = (uint32_t)w[j];
                asm volatile("mad.wide.u32 %0, %1, %2, %0;" : "+l"(w[j]) : "r"(lo), "r"(m));
                lo = (uint32_t)w[(j + 3) & 7];
                asm volatile("mad.wide.u32 %0, %1, %2, %0;" : "+l"(w[j]) : "r"(lo), "r"(m));
            }
        }
        for (int j = 0; j < 8; j++) a[j] = (uint32_t)(w[j] ^ (w[j] >> 32));
    }
    uint32_t x = 0;
    for (int j = 0; j < 16; j++) x ^= a[j];
    if (x == 0x12345678u) sink[blockIdx.x] = x;
}
#endif  // H2B_EXPERIMENTS

template <int IMPL>
__device__ __forceinline__ Fr mul_impl(const Fr& a, const Fr& b)
{
    if (IMPL == 0) return mont_mul_inline<FrCfg>(a, b);
    if (IMPL == 1) return mont_mul_wide<FrCfg>(a, b);
    if (IMPL == 3) return mont_sqr_29<FrCfg>(a);
    if (IMPL == 6) return mont_mul_f64<FrCfg>(a, b);
    return mont_mul_29<FrCfg>(a, b);
}

// Fq products (IMPL 4: a*b 29-bit, 5: a^2 29-bit, 7: a*b FP64).
template <int IMPL>
__global__ void k_fq_mul_batch(const Fq* __restrict__ a, const Fq* __restrict__ b, Fq* __restrict__ out, uint64_t n)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        st(&out[i], IMPL == 4   ? mont_mul_29<FqCfg>(ld(&a[i]), ld(&b[i]))
                    : IMPL == 7 ? mont_mul_f64<FqCfg>(ld(&a[i]), ld(&b[i]))
                                : mont_sqr_29<FqCfg>(ld(&a[i])));
}

// Four independent chains of 29-bit-limb products that stay in limb form.
#if H2B_EXPERIMENTS
__global__ void k_probe_mul29_chain(uint32_t* sink, int iters)
{
    Fr a0 = Fr::one(), b0 = Fr::r2();
    a0.v[0] ^= threadIdx.x;
    Fr m0 = Fr::r2();
    m0.v[2] ^= blockIdx.x;
    Fl<FrCfg> a = to_l(a0), b = to_l(b0), c = to_l(m0), d = to_l(a0), m = to_l(m0);
    for (int it = 0; it < iters; it++) {
        a = mul29(a, m);
        b = mul29(b, m);
        c = mul29(c, m);
        d = mul29(d, m);
    }
    uint32_t x = a.l[0] ^ b.l[1] ^ c.l[2] ^ d.l[3];
    if (x == 0x12345678u) sink[blockIdx.x] = x;
}

template <int IMPL>
__global__ void k_probe_modmul_impl(uint32_t* sink, int iters)
{
    Fr a = Fr::one(), b = Fr::r2(), c = Fr::one(), d = Fr::r2();
    a.v[0] ^= threadIdx.x;
    c.v[1] ^= blockIdx.x;
    Fr m = Fr::r2();
    m.v[2] ^= blockIdx.x;  // not a compile-time constant
    for (int it = 0; it < iters; it++) {
        a = mul_impl<IMPL>(a, m);
        b = mul_impl<IMPL>(b, m);
        c = mul_impl<IMPL>(c, m);
        d = mul_impl<IMPL>(d, m);
    }
    uint32_t x = a.v[0] ^ b.v[1] ^ c.v[2] ^ d.v[3];
    if (x == 0x12345678u) sink[blockIdx.x] = x;
}
#endif  // H2B_EXPERIMENTS

template <int IMPL>
__global__ void k_fr_mul_batch(const Fr* __restrict__ a, const Fr* __restrict__ b, Fr* __restrict__ out, uint64_t n)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        st(&out[i], mul_impl<IMPL>(ld(&a[i]), ld(&b[i])));
}

__global__ void k_probe_modmul(uint32_t* sink, int iters)
{
    Fr a = Fr::one(), b = Fr::r2(), c = Fr::one(), d = Fr::r2();
    a.v[0] ^= threadIdx.x;
    c.v[1] ^= blockIdx.x;
    const Fr m = Fr::r2();
    for (int it = 0; it < iters; it++) {
        a = a * m;
        b = b * m;
        c = c * m;
        d = d * m;
    }
    uint32_t x = a.v[0] ^ b.v[1] ^ c.v[2] ^ d.v[3];
    if (x == 0x12345678u) sink[blockIdx.x] = x;
}

} // namespace h2b

using namespace h2b;

extern "C" void h2b_prof_enable(int on)
{
    std::lock_guard<std::mutex> lk(g_mu);
    for (int i = 0; i < PROF_IDS; i++) {
        for (auto& p : g_used[i]) g_pool.push_back(p);
        g_used[i].clear();
        g_is_open[i] = false;
    }
    g_on = on != 0;
}

// Sums the recorded intervals of `id` (waits for their completion).
extern "C" int h2b_prof_read(int id, double* total_ms, int* count)
{
    if (id < 0 || id >= PROF_IDS) return -1;
    std::lock_guard<std::mutex> lk(g_mu);
    double tot = 0;
    for (auto& p : g_used[id]) {
        cudaEventSynchronize(p.b);
        float ms = 0;
        cudaEventElapsedTime(&ms, p.a, p.b);
        tot += ms;
    }
    *total_ms = tot;
    *count = (int)g_used[id].size();
    return 0;
}

extern "C" RustError h2b_probe_imad(int blocks, int threads, int iters, void* d_sink, cudaStream_t stream)
{
    k_probe_imad<<<blocks, threads, 0, stream>>>((uint32_t*)d_sink, iters, 0x2545f491u);
    H2B_LAUNCHED("k_probe_imad");
    return ok();
}

#if H2B_EXPERIMENTS
extern "C" RustError h2b_probe_imad_form(int blocks, int threads, int iters, int mode, void* d_sink,
                                         cudaStream_t stream)
{
    k_probe_imad_form<<<blocks, threads, 0, stream>>>((uint32_t*)d_sink, iters, 0x2545f491u, mode);
    H2B_LAUNCHED("k_probe_imad_form");
    return ok();
}

// Montgomery-product throughput of one implementation (0 = mad.lo/mad.hi
// carry chains, 1 = mad.wide CIOS, 2 = 29-bit limbs with conversion from and
// to 8 x 32 per product, 3 = 29-bit limbs kept between products, 4 = FP64
// product over 52-bit limbs), four independent products per iteration.
extern "C" RustError h2b_probe_modmul_impl(int impl, int blocks, int threads, int iters, void* d_sink,
                                           cudaStream_t stream)
{
    if (impl == 0) k_probe_modmul_impl<0><<<blocks, threads, 0, stream>>>((uint32_t*)d_sink, iters);
    else if (impl == 1) k_probe_modmul_impl<1><<<blocks, threads, 0, stream>>>((uint32_t*)d_sink, iters);
    else if (impl == 2) k_probe_modmul_impl<2><<<blocks, threads, 0, stream>>>((uint32_t*)d_sink, iters);
    else if (impl == 4) k_probe_modmul_impl<6><<<blocks, threads, 0, stream>>>((uint32_t*)d_sink, iters);
    else k_probe_mul29_chain<<<blocks, threads, 0, stream>>>((uint32_t*)d_sink, iters);
    H2B_LAUNCHED("k_probe_modmul_impl");
    return ok();
}

// out[i] = a[i] * b[i] with the chosen product implementation (tests):
// 0-2 Fr products (CIOS lo/hi, CIOS wide, 29-bit), 3 Fr square (29-bit),
// 4 Fq product, 5 Fq square (29-bit), 6 Fr product, 7 Fq product (FP64).
#endif  // H2B_EXPERIMENTS

extern "C" RustError h2b_fr_mul_batch(int impl, const void* d_a, const void* d_b, void* d_out, uint64_t n,
                                      cudaStream_t stream)
{
    if (n == 0) return ok();
    if (impl == 0)
        k_fr_mul_batch<0><<<grid_for(n, 256), 256, 0, stream>>>((const Fr*)d_a, (const Fr*)d_b, (Fr*)d_out, n);
    else if (impl == 1)
        k_fr_mul_batch<1><<<grid_for(n, 256), 256, 0, stream>>>((const Fr*)d_a, (const Fr*)d_b, (Fr*)d_out, n);
    else if (impl == 2)
        k_fr_mul_batch<2><<<grid_for(n, 256), 256, 0, stream>>>((const Fr*)d_a, (const Fr*)d_b, (Fr*)d_out, n);
    else if (impl == 3)
        k_fr_mul_batch<3><<<grid_for(n, 256), 256, 0, stream>>>((const Fr*)d_a, (const Fr*)d_b, (Fr*)d_out, n);
    else if (impl == 4)
        k_fq_mul_batch<4><<<grid_for(n, 256), 256, 0, stream>>>((const Fq*)d_a, (const Fq*)d_b, (Fq*)d_out, n);
    else if (impl == 6)
        k_fr_mul_batch<6><<<grid_for(n, 256), 256, 0, stream>>>((const Fr*)d_a, (const Fr*)d_b, (Fr*)d_out, n);
    else if (impl == 7)
        k_fq_mul_batch<7><<<grid_for(n, 256), 256, 0, stream>>>((const Fq*)d_a, (const Fq*)d_b, (Fq*)d_out, n);
    else
        k_fq_mul_batch<5><<<grid_for(n, 256), 256, 0, stream>>>((const Fq*)d_a, (const Fq*)d_b, (Fq*)d_out, n);
    H2B_LAUNCHED("k_fr_mul_batch");
    return ok();
}

extern "C" RustError h2b_probe_modmul(int blocks, int threads, int iters, void* d_sink, cudaStream_t stream)
{
    k_probe_modmul<<<blocks, threads, 0, stream>>>((uint32_t*)d_sink, iters);
    H2B_LAUNCHED("k_probe_modmul");
    return ok();
}

extern "C" uint64_t h2b_launch_count(void) { return g_kernel_launches.load(); }
