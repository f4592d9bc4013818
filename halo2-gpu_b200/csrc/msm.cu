// Pippenger G1 MSM behind Params::commit / commit_lagrange
// (halo2_proofs/src/poly/kzg/commitment.rs:456-575) and the reference entry
// points `_halo2_multiexp{,_device_bases,_device_scalars_device_bases}`
// (halo2_proofs/cuda/src/multiexp.cu:260-525, declared at
// halo2_proofs/src/cuda/culib.rs:30-70).
//
// Pipeline (all stream-ordered, no host round trip until the 96-byte result):
//  1. split:   each scalar leaves Montgomery form and is split by the GLV
//              endomorphism into two signed halves below 2^127 (glv.cuh), so
//              n points become 2n virtual points P_i, phi(P_i) with 128-bit
//              scalars: half the windows, half the buckets and half the
//              final doubling chain of a 254-bit Pippenger.  The caller's
//              scalars are never mutated.
//  2. digits:  signed c-bit windows, digits in [-(2^(c-1)-1), 2^(c-1)], so a
//              window needs 2^(c-1) buckets; a negative digit (or a negative
//              half) adds -P.
//  3. sort:    counting sort of (window, bucket) keys -- warp-aggregated
//              histogram, exclusive scan to bucket offsets, warp-aggregated
//              scatter of point indices (sign in bit 31).
//  4. accumulate: the sorted entry list is cut into equal chunks of K entries,
//              one chunk per thread, so dense buckets (e.g. every scalar == 1
//              landing in one bucket) cost the same as sparse ones.  A chunk
//              writes finished buckets directly and the partial sum of the
//              bucket it started in the middle of to a per-chunk slot.
//  5. fixup:   each bucket adds the per-chunk partials it spans; buckets that
//              span many chunks are summed by a CTA-wide tree instead.
//  6. reduce:  per window, buckets are cut into segments; each segment does
//              the running-sum trick and scales by its offset, a CTA tree
//              sums the segments, then 2^(c*w) * W_w is summed over windows.
//  7. output:  XYZZ -> the reference's Jacobian image {x, y, 1} (or (0,1,0)).
#include <algorithm>
#include "abi.cuh"
#include "curve.cuh"
#include "msm.cuh"
#include "prof.cuh"
#include "glv.cuh"
#include "scan_u32.cuh"

extern "C" RustError h2b_exec_fork(cudaStream_t parent, uint32_t n, cudaStream_t* out);  // exec.cu

namespace h2b {

// H2B_EXPERIMENTS=1 also builds the accumulation forms and the batch-affine
// pairing rounds that measured slower than the default (A/B comparisons);
// the shipped library leaves them out.
#ifndef H2B_EXPERIMENTS
#define H2B_EXPERIMENTS 0
#endif
static constexpr int GLV_BITS = 127;
// 32-bit sorted-entry offsets: 2 halves x 8 windows x n < 2^32
static constexpr uint64_t MSM_MAX_LENGTH = 1ull << 27;
static constexpr uint32_t SIGN_BIT = 0x80000000u;
// widest window the tuning override accepts (22 bits: 6 windows per GLV half)
static constexpr int MSM_MAX_WINDOW = 22;
// segment sums per CTA of a bit sum before it is split (reduction step 2)
static constexpr uint32_t BITSUM_ITEMS = 4096;
static constexpr uint32_t DENSE_LIMIT = 32;     // chunks per bucket summed serially in fixup
static constexpr int DENSE_PIECES = 32;          // CTAs per dense bucket
static constexpr uint64_t ACC_TARGET_CHUNKS = 148ull * 3 * 128 * 4;  // accumulation threads x 4
static constexpr uint64_t ACC_MIN_K = 16;       // smallest chunk of the default plan
static constexpr uint64_t MSM_PIPE_MIN = 1ull << 18;  // host scalars from here on are copied in pieces
static constexpr int MSM_PIPE_PIECES = 8;

static int g_msm_window_override = 0;
static int g_msm_acc_variant = 6;  // form and call structure of the accumulation kernel (0..6)
static int g_msm_pair_rounds = 0;  // batch-affine pairing rounds before the XYZZ accumulation (0..3)
constexpr int PR_T = 128;          // pairing rounds: threads per CTA
constexpr int PR_E = 8;            // pairing rounds: input entries per thread (at most 4 additions)
static uint64_t pr_ctas(uint64_t entries) { return (entries + (uint64_t)PR_T * PR_E - 1) / ((uint64_t)PR_T * PR_E); }

uint64_t fq_batch_invert_scratch(uint64_t n);
int tune_value(int param, int log_n);  // tune.cu
RustError fq_batch_invert(Fq* d, uint64_t n, void* scratch, uint64_t scratch_bytes, cudaStream_t st);

void msm_set_pair_rounds(int rounds)
{
    if (rounds >= 0 && rounds <= (H2B_EXPERIMENTS ? 3 : 0)) g_msm_pair_rounds = rounds;
}
static int g_msm_chunk_override = 0;
static uint32_t g_msm_prefetch = 2;   // entries ahead whose point the accumulation prefetches into L2 (0: none)

void msm_set_tuning(int window_bits, int chunk)
{
    g_msm_window_override = window_bits;
    g_msm_chunk_override = chunk;
}

static int floor_log2(uint64_t n)
{
    int lg = 0;
    while ((1ull << (lg + 1)) <= n) lg++;
    return lg;
}

// `plain`: an MSM over plain bases, whose window width may come from the
// per-size tuning table; a window table's width is fixed when it is built.
static int choose_c(uint64_t n, bool plain = false)
{
    const int lg = floor_log2(n);
    if (g_msm_window_override >= 4 && g_msm_window_override <= MSM_MAX_WINDOW) return g_msm_window_override;
    if (plain) {
        const int tuned = tune_value(0, lg);
        if (tuned) return tuned;
        // plain-base widths from autotuner runs on B200 (witness-like scalar
        // mix): 16 bits from 2^20 (5.40 -> 4.36 ms with the chunk rule below),
        // 13 bits from 2^14 (2^16: 1.79 -> 1.45 ms); 17 to 20 bits measured
        // slower from 2^20 to 2^22 (2^22: 11.30 ms at 16, 13.4-19.6 ms wider)
        if (lg >= 20) return 16;
        if (lg >= 19) return 15;
        if (lg >= 14) return 13;
        if (lg >= 10) return 10;
        return 7;
    }
    // Window tables: every window's digits land in one bucket set of 2^(c-1)
    // buckets, so a narrow window makes few, long buckets (2^18 points at 13
    // bits: 4096 buckets of about 1300 entries).
    // Widths from a sweep of c in 10..18 on B200 (bench.py --case
    // table_widths; uniform / witness-mix scalars, n = table size): 2^18
    // table 11.57 / 3.07 ms at 13 bits -> 1.80 / 1.48 ms at 16, 2^20 6.32 /
    // 4.64 ms at 15 -> 4.91 / 3.46 ms at 16, 2^16 4.48 / 1.20 ms at 12 ->
    // 1.02 / 0.85 ms at 13.
    if (lg >= 17) return 16;
    if (lg >= 13) return 13;
    if (lg >= 10) return 10;
    return 7;
}

// tn > 0: precomputed window table of tn points per window; all windows then
// share one bucket set and the reduction has a single window.
static MsmPlan plan_core(uint64_t n, int c, uint64_t tn, uint32_t concurrent = 1)
{
    MsmPlan p;
    p.n = n;
    p.tn = tn;
    p.c = c;
    // GLV halves: magnitudes < 2^GLV_BITS; the top window must leave room
    // for the signed-digit carry (its width <= c - 1).
    p.W = (GLV_BITS + c - 1) / c;
    if (GLV_BITS - c * (p.W - 1) > c - 1) p.W++;
    p.H = 1u << (c - 1);
    p.Wr = tn ? 1 : p.W;
    p.NB = (uint64_t)p.Wr * p.H;
    p.nv = 2 * n;
    p.max_entries = p.nv * (uint64_t)p.W;
    // Entries per accumulation chunk (one thread walks a chunk): 128 when the
    // entries give at least ACC_TARGET_CHUNKS chunks (k >= 20 at every
    // window size), fewer for a small MSM so that about ACC_TARGET_CHUNKS
    // threads still run (148 SMs x 3 CTAs x 128 threads, 4 chunks each).
    // MSMs that run `concurrent` at a time share that target.  A smaller K
    // adds chunk heads that the fixup sums serially per bucket, so K must
    // not drop where buckets are long: on the 64-job batch (16 streams) a
    // fixed K = 32 took 133 ms over a window table against 85 ms at 128.
    const uint64_t k_fit = p.max_entries / std::max<uint64_t>(1, ACC_TARGET_CHUNKS / std::max(concurrent, 1u));
    // A tuned chunk size applies to an MSM that runs alone (batched MSMs keep
    // the formula, which accounts for the MSMs running beside them).
    // A plain-base MSM that runs alone takes half the fitted chunk, at most
    // 64 (B200 autotuner runs: 2^22 128 -> 64 entries 11.89 -> 11.45 ms;
    // 2^20 at 16 bits chose 32 entries): twice the chunks hide more of the
    // accumulation's latency than the extra chunk heads cost the fixup.  Not
    // over a window table: its single bucket set holds W times longer
    // buckets, which at 64 entries span more than DENSE_LIMIT chunks and take
    // the dense path (k = 22 prover-shaped proof 398 -> 438 ms).
    const bool alone_plain = concurrent <= 1 && tn == 0;
    const int tuned_k = alone_plain ? tune_value(1, floor_log2(n)) : 0;
    const uint64_t k_rule = alone_plain ? std::min<uint64_t>(64, std::max<uint64_t>(ACC_MIN_K, k_fit / 2))
                                        : std::min<uint64_t>(128, std::max<uint64_t>(ACC_MIN_K, k_fit));
    p.K = g_msm_chunk_override > 0 ? (uint32_t)g_msm_chunk_override
          : tuned_k > 0            ? (uint32_t)tuned_k
                                   : (uint32_t)k_rule;
    // pairing rounds: round r leaves at most cap[r-1]/2 + NB/2 entries
    p.R = tn ? 0 : g_msm_pair_rounds;
    p.cap[0] = p.max_entries;
    for (int r = 1; r <= 3; r++) p.cap[r] = p.cap[r - 1] / 2 + p.NB / 2 + 1;
    p.Kf = p.R > 0 ? std::max<uint32_t>(8u, p.K >> p.R) : p.K;
    const uint64_t final_entries = p.cap[p.R];
    p.max_chunks = (final_entries + p.Kf - 1) / p.Kf + 1;
    // segments per window for the running-sum reduction (L buckets each)
    uint32_t L = p.H >= 256 ? 8u : (p.H >= 4 ? 4u : 1u);
    p.L = L;
    p.LOGL = 31 - __builtin_clz(L);
    p.S = p.H / L;
    p.NBITS = p.S > 1 ? 31 - __builtin_clz(p.S) : 0;
    // a bit sum of more than BITSUM_ITEMS segment sums is split over CTAs
    // (wide windows over a table: one bucket set of 2^(c-1) buckets, a
    // single reduction window, so only NBITS + 1 bit sums to spread)
    p.BP = std::max<uint32_t>(1u, (p.S + BITSUM_ITEMS - 1) / BITSUM_ITEMS);
    // a bucket spanning more than DENSE_LIMIT chunks holds > DENSE_LIMIT*K entries
    p.max_dense = final_entries / ((uint64_t)DENSE_LIMIT * p.Kf) + 1;
    return p;
}

MsmPlan msm_plan(uint64_t n) { return plan_core(n, choose_c(n, true), 0); }

MsmPlan msm_plan_table(uint64_t n, uint64_t tn) { return plan_core(n, choose_c(tn), tn); }

MsmPlan msm_plan_shared(uint64_t n, uint64_t tn, uint32_t concurrent)
{
    return tn ? plan_core(n, choose_c(tn), tn, concurrent) : plan_core(n, choose_c(n, true), 0, concurrent);
}

// J MSMs over one window table of tn points, n_total scalars in all, as one
// run: job j's entries go to bucket set j (J bucket sets of H buckets), so
// the sort, the accumulation and the bucket reduction run once for all jobs.
MsmPlan msm_plan_merged(uint64_t n_total, uint64_t tn, uint32_t J)
{
    MsmPlan p = plan_core(n_total, choose_c(tn), tn);
    p.Wr = (int)J;
    p.NB = (uint64_t)J * p.H;
    return p;
}

void msm_plan_scratch(const MsmPlan& p, ScratchPlan& sp, bool scalar_host, bool bases_host)
{
    if (bases_host) sp.add(p.n * sizeof(G1Affine));
    if (scalar_host) sp.add(p.n * sizeof(Fr));       // host scalars staged here
    sp.add(p.n * sizeof(Fr));                         // canonical scalars
    sp.add_n<uint32_t>(p.NB);                         // counts
    sp.add_n<uint32_t>(p.NB + 1);                     // offsets
    sp.add_n<uint32_t>(p.NB);                         // cursor
    sp.add_n<uint32_t>(scan_u32_tiles(p.NB) + 1);     // scan tiles
    sp.add_n<uint32_t>(p.max_entries);                // sorted entries
    sp.add_n<G1Xyzz>(p.NB);                           // bucket sums
    sp.add_n<G1Xyzz>(p.max_chunks);                   // chunk head partials
    sp.add_n<uint32_t>(p.max_dense + 1);              // dense list + count
    sp.add_n<G1Xyzz>(p.max_dense * DENSE_PIECES);     // dense pieces
    sp.add_n<G1Xyzz>((uint64_t)p.Wr * p.S);           // segment weighted sums
    sp.add_n<G1Xyzz>((uint64_t)p.Wr * p.S);           // segment plain sums
    sp.add_n<G1Xyzz>((uint64_t)std::max(p.W, p.Wr) * (p.NBITS + 1));  // per-bit sums
    if (p.BP > 1) sp.add_n<G1Xyzz>((uint64_t)p.Wr * (p.NBITS + 1) * p.BP);  // their parts
    sp.add_n<G1Xyzz>(std::max(p.W, p.Wr));                            // window sums
    sp.add_n<G1Jac>(1);                               // result
    if (p.R >= 1) sp.add_n<G1Affine>(p.cap[1]);       // round outputs 1, 3
    if (p.R >= 2) sp.add_n<G1Affine>(p.cap[2]);       // round output 2
    for (int r = 0; r < p.R; r++) sp.add_n<uint32_t>(p.NB + 1);  // round offsets
    if (p.R >= 1) {                                   // sized for round 1, reused by later rounds
        const uint64_t ctas = pr_ctas(p.cap[0]);
        sp.add_n<Fq>(ctas * PR_T * 4);                // denominator prefixes
        sp.add_n<uint2>(ctas * PR_T * 4);             // jobs
        sp.add_n<uint32_t>(ctas * PR_T);              // jobs per thread
        sp.add_n<Fq>(ctas * 2 * PR_T);                // product trees
        sp.add_n<Fq>(ctas);                           // CTA totals
        sp.add(fq_batch_invert_scratch(ctas));
    }
    if (p.tn == 0 && p.R == 0) sp.add_n<G1Affine>(2 * p.n);  // P_i and phi(P_i) in the lazy form (x 2^261)
}

MsmScratch msm_carve(const MsmPlan& p, ScratchArena& ar, bool scalar_host, bool bases_host)
{
    MsmScratch s;
    s.bases_stage = bases_host ? (G1Affine*)ar.take(p.n * sizeof(G1Affine)) : nullptr;
    s.scalar_stage = scalar_host ? (Fr*)ar.take(p.n * sizeof(Fr)) : nullptr;
    s.canon = (Fr*)ar.take(p.n * sizeof(Fr));
    s.counts = ar.take_n<uint32_t>(p.NB);
    s.offsets = ar.take_n<uint32_t>(p.NB + 1);
    s.cursor = ar.take_n<uint32_t>(p.NB);
    s.scan_tmp = ar.take_n<uint32_t>(scan_u32_tiles(p.NB) + 1);
    s.sorted = ar.take_n<uint32_t>(p.max_entries);
    s.buckets = ar.take_n<G1Xyzz>(p.NB);
    s.heads = ar.take_n<G1Xyzz>(p.max_chunks);
    s.dense = ar.take_n<uint32_t>(p.max_dense + 1);
    s.pieces = ar.take_n<G1Xyzz>(p.max_dense * DENSE_PIECES);
    s.segacc = ar.take_n<G1Xyzz>((uint64_t)p.Wr * p.S);
    s.segrun = ar.take_n<G1Xyzz>((uint64_t)p.Wr * p.S);
    s.bits = ar.take_n<G1Xyzz>((uint64_t)std::max(p.W, p.Wr) * (p.NBITS + 1));
    s.bitparts = p.BP > 1 ? ar.take_n<G1Xyzz>((uint64_t)p.Wr * (p.NBITS + 1) * p.BP) : nullptr;
    s.wins = ar.take_n<G1Xyzz>(std::max(p.W, p.Wr));
    s.result = ar.take_n<G1Jac>(1);
    s.pts[0] = p.R >= 1 ? ar.take_n<G1Affine>(p.cap[1]) : nullptr;
    s.pts[1] = p.R >= 2 ? ar.take_n<G1Affine>(p.cap[2]) : nullptr;
    for (int r = 0; r < 3; r++) s.roff[r] = r < p.R ? ar.take_n<uint32_t>(p.NB + 1) : nullptr;
    s.pr_pref = nullptr; s.pr_job = nullptr; s.pr_nj = nullptr; s.pr_tree = nullptr; s.pr_tot = nullptr;
    s.pr_inv_scratch = nullptr; s.pr_inv_bytes = 0;
    if (p.R >= 1) {
        const uint64_t ctas = pr_ctas(p.cap[0]);
        s.pr_pref = ar.take_n<Fq>(ctas * PR_T * 4);
        s.pr_job = ar.take_n<uint2>(ctas * PR_T * 4);
        s.pr_nj = ar.take_n<uint32_t>(ctas * PR_T);
        s.pr_tree = ar.take_n<Fq>(ctas * 2 * PR_T);
        s.pr_tot = ar.take_n<Fq>(ctas);
        s.pr_inv_bytes = fq_batch_invert_scratch(ctas);
        s.pr_inv_scratch = ar.take(s.pr_inv_bytes);
    }
    s.rbases = (p.tn == 0 && p.R == 0) ? ar.take_n<G1Affine>(2 * p.n) : nullptr;
    return s;
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------

// Virtual scalars: vs[2i] = k1, vs[2i+1] = k2 of the GLV split of scalar i
// (128-bit magnitudes, sign in bit 127), so entry v stands for point i = v/2,
// taken as P_i (v even) or phi(P_i) (v odd).
// GLV split of each scalar; with `rb` set, base i is also converted to the
// lazy x 2^261 form the accumulation reads (same index space, one launch):
// rb[i] = P_i and rb[n + i] = phi(P_i) = (beta x, y), so the accumulation
// multiplies by beta nowhere.
__global__ void k_msm_glv(const Fr* __restrict__ sc, uint4* __restrict__ vs, uint64_t lo, uint64_t hi,
                          const G1Affine* __restrict__ bases, G1Affine* __restrict__ rb, uint64_t n)
{
    const Fq beta = glv::beta();
    for (uint64_t i = lo + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < hi;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint4 a, b;
        glv::decompose(from_mont(ldg(&sc[i])), a, b);
        vs[2 * i] = a;
        vs[2 * i + 1] = b;
        if (rb) {
            const G1Affine q = ld_affine(&bases[i]);
            const Fq y = to_r261(q.y);
            st(&rb[i].x, to_r261(q.x));
            st(&rb[i].y, y);
            st(&rb[n + i].x, to_r261(q.x * beta));     // infinity (0, 0) stays (0, 0)
            st(&rb[n + i].y, y);
        }
    }
}

__device__ __forceinline__ uint32_t window_bits(const uint4& s, int bit, int c)
{
    const uint32_t w[5] = {s.x, s.y, s.z, s.w & 0x7fffffffu, 0u};
    int li = bit >> 5, sh = bit & 31;
    uint64_t v = ((uint64_t)w[li] | ((uint64_t)w[li + 1] << 32)) >> sh;
    return (uint32_t)(v & ((1ull << c) - 1));
}

// Signed digit w of a virtual scalar (carry in/out through `carry`) and its
// bucket key w*H + |d| - 1, or ~0 for a zero digit or an invalid lane.
// With a window table every window shares one bucket set, based at `kb`
// (the job's bucket set in a merged run, 0 otherwise).  The histogram and
// the scatter both take their keys from here, so their counts agree.
__device__ __forceinline__ uint32_t digit_key(const uint4& s, int w, int c, uint32_t H, uint32_t& carry, bool valid,
                                              uint64_t tn, uint32_t kb, int32_t& d)
{
    const uint32_t v = window_bits(s, w * c, c) + carry;
    if (v > H) { d = (int32_t)v - (int32_t)(1u << c); carry = 1; }
    else { d = (int32_t)v; carry = 0; }
    return (valid && d != 0) ? (tn ? kb : (uint32_t)w * H) + (uint32_t)(d < 0 ? -d : d) - 1u : 0xffffffffu;
}

// Warp-aggregated count of one key per lane (all 32 lanes call it together).
__device__ __forceinline__ void hist_key(uint32_t key, uint32_t* __restrict__ counts)
{
    const unsigned lane = threadIdx.x & 31;
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    if (key != 0xffffffffu && (int)lane == __ffs(peers) - 1) atomicAdd(&counts[key], __popc(peers));
}

// For each digit: key = w*H + |d| - 1 (or ~0 for zero digits); the entry's
// sign is the digit's sign flipped by the virtual scalar's sign.
// Virtual points v0 <= i < n.
template <bool SCATTER>
__global__ void k_msm_sort(const uint4* __restrict__ vsc, uint64_t v0, uint64_t n, int c, int W, uint32_t H,
                           uint32_t* __restrict__ counts_or_cursor, uint32_t* __restrict__ sorted, uint64_t tn,
                           uint32_t kb)
{
    const unsigned lane = threadIdx.x & 31;
    for (uint64_t base = v0 + blockIdx.x * (uint64_t)blockDim.x; base < n; base += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t i = base + threadIdx.x;
        bool valid = i < n;
        uint4 s = valid ? vsc[i] : make_uint4(0u, 0u, 0u, 0u);
        const bool sneg = (s.w >> 31) != 0;
        uint32_t carry = 0;
        for (int w = 0; w < W; w++) {
            int32_t d;
            const uint32_t key = digit_key(s, w, c, H, carry, valid, tn, kb, d);
            unsigned peers = __match_any_sync(0xffffffffu, key);
            int leader = __ffs(peers) - 1;
            if (!SCATTER) {
                if (key != 0xffffffffu && (int)lane == leader) atomicAdd(&counts_or_cursor[key], __popc(peers));
            } else {
                uint32_t b = 0;
                if (key != 0xffffffffu && (int)lane == leader) b = atomicAdd(&counts_or_cursor[key], __popc(peers));
                b = __shfl_sync(0xffffffffu, b, leader);
                if (key != 0xffffffffu) {
                    uint32_t rank = __popc(peers & ((1u << lane) - 1u));
                    // with a window table the entry names table point w * tn + i/2
                    const uint32_t v = (uint32_t)(i + 2 * (uint64_t)w * tn);
                    sorted[b + rank] = v | (((d < 0) != sneg) ? SIGN_BIT : 0u);
                }
            }
        }
    }
}

// The GLV split and base conversion of k_msm_glv fused with the digit
// histogram of k_msm_sort<false> for the two halves of each scalar: the
// histogram's atomics overlap the split's memory traffic, and the halves are
// counted from registers instead of re-read.  Loops are block-uniform so
// that every lane reaches the warp-wide match.
__global__ void k_msm_glv_hist(const Fr* __restrict__ sc, uint4* __restrict__ vs, uint64_t lo, uint64_t hi,
                               const G1Affine* __restrict__ bases, G1Affine* __restrict__ rb, uint64_t n, int c,
                               int W, uint32_t H, uint32_t* __restrict__ counts, uint64_t tn)
{
    const Fq beta = glv::beta();
    for (uint64_t base = lo + blockIdx.x * (uint64_t)blockDim.x; base < hi; base += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i = base + threadIdx.x;
        const bool valid = i < hi;
        uint4 a = make_uint4(0u, 0u, 0u, 0u), b = a;
        if (valid) {
            glv::decompose(from_mont(ldg(&sc[i])), a, b);
            vs[2 * i] = a;
            vs[2 * i + 1] = b;
            if (rb) {
                const G1Affine q = ld_affine(&bases[i]);
                const Fq y = to_r261(q.y);
                st(&rb[i].x, to_r261(q.x));
                st(&rb[i].y, y);
                st(&rb[n + i].x, to_r261(q.x * beta));     // infinity (0, 0) stays (0, 0)
                st(&rb[n + i].y, y);
            }
        }
        uint32_t ca = 0, cb = 0;
        for (int w = 0; w < W; w++) {
            int32_t d;
            hist_key(digit_key(a, w, c, H, ca, valid, tn, 0u, d), counts);
            hist_key(digit_key(b, w, c, H, cb, valid, tn, 0u, d), counts);
        }
    }
}

#if H2B_EXPERIMENTS
// One thread per chunk of K sorted entries; the running bucket sum stays in
// 29-bit limb form and is packed to the canonical 8 x 32 image when stored.
// PTS: the entries are the affine points themselves (bases[e]), as left by
// the pairing rounds, instead of signed (GLV) indices into the bases.
template <int MODE, bool PTS>
__global__ void __launch_bounds__(128, MODE == 1 ? 2 : (MODE >= 3 ? MODE + 1 : 3)) k_msm_accumulate(const uint32_t* __restrict__ sorted,
                                                        const uint32_t* __restrict__ offsets, uint64_t NB, uint32_t K,
                                                        const G1Affine* __restrict__ bases, G1Xyzz* __restrict__ buckets,
                                                        G1Xyzz* __restrict__ heads)
{
    const uint32_t M = offsets[NB];
    const uint64_t nchunks = (M + (uint64_t)K - 1) / K;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < nchunks;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t start = (uint32_t)(t * K);
        const uint32_t end = ((uint64_t)start + K < (uint64_t)M) ? start + K : M;
        uint64_t lo = 0, hi = NB;  // offsets[lo] <= start < offsets[hi]
        while (hi - lo > 1) {
            uint64_t mid = (lo + hi) >> 1;
            if (offsets[mid] <= start) lo = mid; else hi = mid;
        }
        uint64_t b = lo;
        uint32_t next = offsets[b + 1];
        bool head = offsets[b] < start;
        G1XyzzL acc = xyzzl_inf();
        for (uint32_t e = start; e < end; e++) {
            if (e == next) {
                if (head) st_xyzz(&heads[t], xyzzl_to(acc)); else st_xyzz(&buckets[b], xyzzl_to(acc));
                acc = xyzzl_inf();
                head = false;
                do { b++; next = offsets[b + 1]; } while (next == e);
            }
            if (PTS) {  // contiguous affine points left by the pairing rounds
                const G1Affine P = ld_affine(&bases[e]);
                if (is_inf(P)) continue;
                xyzzl_madd<MODE>(acc, to_l(P.x), to_l(P.y));
                continue;
            }
            const uint32_t ent = sorted[e];
            const uint32_t v = ent & ~SIGN_BIT;
            G1Affine P = ld_affine(&bases[v >> 1]);
            if (is_inf(P)) continue;
            if (ent & SIGN_BIT) P.y = fneg(P.y);
            FqL qx = to_l(P.x);
            if (v & 1u) qx = fl_mul(qx, to_l(glv::beta()));  // phi(P)
            xyzzl_madd<MODE>(acc, qx, to_l(P.y));
        }
        if (head) st_xyzz(&heads[t], xyzzl_to(acc)); else st_xyzz(&buckets[b], xyzzl_to(acc));
    }
}

#endif  // H2B_EXPERIMENTS

// Bases (affine, memory image x 2^256 mod p) -> canonical x 2^261 mod p, the
// form the lazy accumulation reads; infinity (0, 0) stays (0, 0).
__global__ void k_to_r261(const G1Affine* in, G1Affine* out, uint64_t n, G1Affine* phi)  // in may equal out
{
    const Fq beta = glv::beta();
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const G1Affine a = ld_affine(&in[i]);
        G1Affine r;
        r.x = to_r261(a.x);
        r.y = to_r261(a.y);
        if (phi) {
            st(&phi[i].x, to_r261(a.x * beta));   // phi(P) = (beta x, y); infinity stays (0, 0)
            st(&phi[i].y, r.y);
        }
        st(&out[i].x, r.x);
        st(&out[i].y, r.y);
    }
}

// The accumulation in the lazy form (curve.cuh, lazy.cuh): same chunking,
// bucket boundaries and outputs as k_msm_accumulate, over bases in the
// x 2^261 form.  The accumulator's additions and subtractions are one-step
// carry passes with no conditional correction; results are converted back
// to the canonical memory image when a bucket or chunk head is stored.
// phi(P) of the point at bases[j] is stored at bases[phi_off + j] (plain
// bases: phi_off = n; window tables: W n, after all slices).
__global__ void __launch_bounds__(128, 3) k_msm_accumulate_z(const uint32_t* __restrict__ sorted,
                                                             const uint32_t* __restrict__ offsets, uint64_t NB,
                                                             uint32_t K, const G1Affine* __restrict__ bases,
                                                             uint64_t phi_off, G1Xyzz* __restrict__ buckets,
                                                             G1Xyzz* __restrict__ heads)
{
    const FqZ one = fz_from_words(to_r261(Fq::one()));           // 1 in the lazy form (2^261 mod p)
    const FqZ r256 = fz_from_words(Fq::one());                    // 2^256 mod p, for the stores
    const uint32_t M = offsets[NB];
    const uint64_t nchunks = (M + (uint64_t)K - 1) / K;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < nchunks;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t start = (uint32_t)(t * K);
        const uint32_t end = ((uint64_t)start + K < (uint64_t)M) ? start + K : M;
        uint64_t lo = 0, hi = NB;  // offsets[lo] <= start < offsets[hi]
        while (hi - lo > 1) {
            uint64_t mid = (lo + hi) >> 1;
            if (offsets[mid] <= start) lo = mid; else hi = mid;
        }
        uint64_t b = lo;
        uint32_t next = offsets[b + 1];
        bool head = offsets[b] < start;
        G1XyzzZ acc = xyzzz_inf();
        for (uint32_t e = start; e < end; e++) {
            if (e == next) {
                st_xyzzz(head ? &heads[t] : &buckets[b], acc, r256);
                acc = xyzzz_inf();
                head = false;
                do { b++; next = offsets[b + 1]; } while (next == e);
            }
            const uint32_t ent = sorted[e];
            const uint32_t v = ent & ~SIGN_BIT;
            const bool phi = (v & 1u) != 0;
            const G1Affine P = ld_affine(&bases[(v >> 1) + (phi ? phi_off : 0)]);    // phi(P) precomputed
            if (is_inf(P)) continue;
            FqZ qx = fz_from_words(P.x);                                   // < p
            FqZ qy = fz_from_words(P.y);                                   // < p
            if (ent & SIGN_BIT) qy = fz_sub<FqCfg, 2>(fz_zero<FqCfg>(), qy);  // 2p - y < 2p

            xyzzz_madd(acc, qx, qy, one);
        }
        st_xyzzz(head ? &heads[t] : &buckets[b], acc, r256);
    }
}

// The same accumulation in the FP64 lazy form (R' = 2^260, lazy64.cuh):
// bases are read in the same x 2^261 storage form and halved modulo p on
// load; buckets leave in the same canonical memory image.
__global__ void __launch_bounds__(128, 3) k_msm_accumulate_d(const uint32_t* __restrict__ sorted,
                                                             const uint32_t* __restrict__ offsets, uint64_t NB,
                                                             uint32_t K, const G1Affine* __restrict__ bases,
                                                             uint64_t phi_off, G1Xyzz* __restrict__ buckets,
                                                             G1Xyzz* __restrict__ heads, uint32_t pf)
{
    const uint32_t M = offsets[NB];
    const uint64_t nchunks = (M + (uint64_t)K - 1) / K;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < nchunks;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t start = (uint32_t)(t * K);
        const uint32_t end = ((uint64_t)start + K < (uint64_t)M) ? start + K : M;
        uint64_t lo = 0, hi = NB;  // offsets[lo] <= start < offsets[hi]
        while (hi - lo > 1) {
            uint64_t mid = (lo + hi) >> 1;
            if (offsets[mid] <= start) lo = mid; else hi = mid;
        }
        uint64_t b = lo;
        uint32_t next = offsets[b + 1];
        bool head = offsets[b] < start;
        G1XyzzD acc = xyzzd_inf();
        for (uint32_t e = start; e < end; e++) {
            if (e == next) {
                st_xyzzd(head ? &heads[t] : &buckets[b], acc);
                acc = xyzzd_inf();
                head = false;
                do { b++; next = offsets[b + 1]; } while (next == e);
            }
            if (pf && e + pf < end) {   // bring the point pf entries ahead into L2 (no registers held)
                const uint32_t vn = sorted[e + pf] & ~SIGN_BIT;
                const G1Affine* pn = &bases[(vn >> 1) + ((vn & 1u) ? phi_off : 0)];
                asm volatile("prefetch.global.L2 [%0];" ::"l"(pn));
            }
            const uint32_t ent = sorted[e];
            const uint32_t v = ent & ~SIGN_BIT;
            const bool phi = (v & 1u) != 0;
            const G1Affine P = ld_affine(&bases[(v >> 1) + (phi ? phi_off : 0)]);    // phi(P) precomputed
            if (is_inf(P)) continue;
            const FqD qx = fd_from_r261(P.x);                              // < p
            FqD qy = fd_from_r261(P.y);                                    // < p
            if (ent & SIGN_BIT) qy = fd_sub<FqCfg, 2>(fd_zero<FqCfg>(), qy);  // 2p - y < 2p
            xyzzd_madd(acc, qx, qy);
        }
        st_xyzzd(head ? &heads[t] : &buckets[b], acc);
    }
}

#if H2B_EXPERIMENTS
// The FP64 lazy accumulation with two independent chains per thread: the
// entries of a bucket segment alternate between two accumulators whose
// additions share their out-of-line product calls (xyzzd_madd_x2), and the
// two are added once when the segment's bucket (or chunk head) is stored.
// Same chunks, bucket boundaries and outputs as k_msm_accumulate_d.  Measured
// at 2^22 with the witness mix: 25.7 ms against 11.4 ms (255 registers and
// spills halve the warps per SM; the second chain does not make up for it).
__global__ void __launch_bounds__(128, 2) k_msm_accumulate_d2(const uint32_t* __restrict__ sorted,
                                                              const uint32_t* __restrict__ offsets, uint64_t NB,
                                                              uint32_t K, const G1Affine* __restrict__ bases,
                                                              uint64_t phi_off, G1Xyzz* __restrict__ buckets,
                                                              G1Xyzz* __restrict__ heads)
{
    const uint32_t M = offsets[NB];
    const uint64_t nchunks = (M + (uint64_t)K - 1) / K;
    auto load = [&](uint32_t e, FqD& qx, FqD& qy) -> bool {    // false for a point at infinity
        const uint32_t ent = sorted[e];
        const uint32_t v = ent & ~SIGN_BIT;
        const G1Affine P = ld_affine(&bases[(v >> 1) + ((v & 1u) ? phi_off : 0)]);
        if (is_inf(P)) return false;
        qx = fd_from_r261(P.x);                                        // < p
        qy = fd_from_r261(P.y);                                        // < p
        if (ent & SIGN_BIT) qy = fd_sub<FqCfg, 2>(fd_zero<FqCfg>(), qy);  // 2p - y < 2p
        return true;
    };
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < nchunks;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t start = (uint32_t)(t * K);
        const uint32_t end = ((uint64_t)start + K < (uint64_t)M) ? start + K : M;
        uint64_t lo = 0, hi = NB;  // offsets[lo] <= start < offsets[hi]
        while (hi - lo > 1) {
            uint64_t mid = (lo + hi) >> 1;
            if (offsets[mid] <= start) lo = mid; else hi = mid;
        }
        uint64_t b = lo;
        uint32_t next = offsets[b + 1];
        bool head = offsets[b] < start;
        G1XyzzD a0 = xyzzd_inf(), a1 = xyzzd_inf();
        uint32_t e = start;
        while (e < end) {
            if (e == next) {
                st_xyzzd_pair(head ? &heads[t] : &buckets[b], a0, a1);
                a0 = xyzzd_inf();
                a1 = xyzzd_inf();
                head = false;
                do { b++; next = offsets[b + 1]; } while (next == e);
            }
            const uint32_t seg = next < end ? next : end;
            for (; e + 1 < seg; e += 2) {
                FqD x0, y0, x1, y1;
                const bool f0 = load(e, x0, y0), f1 = load(e + 1, x1, y1);
                if (f0 && f1) {
                    xyzzd_madd_x2(a0, x0, y0, a1, x1, y1);
                } else {
                    if (f0) xyzzd_madd(a0, x0, y0);
                    if (f1) xyzzd_madd(a1, x1, y1);
                }
            }
            if (e < seg) {
                FqD x0, y0;
                if (load(e, x0, y0)) xyzzd_madd(a0, x0, y0);
                e++;
            }
        }
        st_xyzzd_pair(head ? &heads[t] : &buckets[b], a0, a1);
    }
}

// ---- pairing rounds (batch-affine bucket additions) -----------------------
// Round r adds the points of every bucket pairwise in affine coordinates:
// entries (2j, 2j+1) of a bucket become output point j (an odd last entry is
// copied), so each round halves every bucket.  lambda = (y2 - y1) / (x2 - x1)
// (or 3 x1^2 / (2 y1) for equal points) needs one inversion per addition; all
// denominators share inversions through Montgomery's trick, so an addition
// costs about 6 products against 10 for an XYZZ mixed addition, and the
// additions of a thread are independent of each other.  Infinity inputs pass
// the other point through; P + (-P) gives infinity, written as (0, 0) like an
// input base.  A round is three launches: forward products with a product
// tree per CTA, one batch inversion of all CTA totals, backward pass.  (An
// inversion inside each CTA would put a long serial binary GCD behind every
// 512 additions.)

__device__ __forceinline__ void st_affine(G1Affine* p, const G1Affine& a)
{
    st(&p->x, a.x);
    st(&p->y, a.y);
}

template <bool FIRST>
__device__ __forceinline__ G1Affine pr_load(const uint32_t* __restrict__ sorted, const G1Affine* __restrict__ src,
                                            uint32_t e)
{
    if (!FIRST) return ld_affine(&src[e]);
    const uint32_t ent = sorted[e];
    const uint32_t v = ent & ~SIGN_BIT;
    G1Affine P = ld_affine(&src[v >> 1]);
    if (is_inf(P)) return P;
    if (v & 1u) P.x = P.x * glv::beta();  // phi(P)
    if (ent & SIGN_BIT) P.y = fneg(P.y);
    return P;
}

// Denominator and numerator of lambda for P1 + P2 (both finite, P2 != -P1).
__device__ __forceinline__ void pr_slope_terms(const G1Affine& P1, const G1Affine& P2, FqL& d, FqL& num)
{
    const FqL x1 = to_l(P1.x), y1 = to_l(P1.y);
    if (P1.x != P2.x) {
        d = fl_sub(to_l(P2.x), x1);
        num = fl_sub(to_l(P2.y), y1);
    } else {
        d = fl_add(y1, y1);
        const FqL xx = fl_sqr(x1);
        num = fl_add(fl_add(xx, xx), xx);
    }
}

// Forward half.  A thread owns PR_E input entries; every entry at an even
// position of its bucket starts an addition with the next entry (at most 4
// per thread).  Running products of the denominators go to g_pref, the jobs
// to g_job / g_nj, the CTA's product tree over the thread totals to g_tree
// (nodes 1 .. 2T-1) and its root to g_tot[cta].  CTAs past the last entry
// only set g_tot[cta] = 1.
template <bool FIRST>
__global__ void __launch_bounds__(PR_T) k_msm_pair_fwd(const uint32_t* __restrict__ sorted,
                                                       const G1Affine* __restrict__ src,
                                                       const uint32_t* __restrict__ in_off, uint64_t NB,
                                                       const uint32_t* __restrict__ out_off,
                                                       G1Affine* __restrict__ out_pts, Fq* __restrict__ g_pref,
                                                       uint2* __restrict__ g_job, uint32_t* __restrict__ g_nj,
                                                       Fq* __restrict__ g_tree, Fq* __restrict__ g_tot)
{
    __shared__ FqL tree[2 * PR_T];
    const int t = threadIdx.x;
    const uint32_t M = in_off[NB];
    const uint64_t cta = blockIdx.x;
    const uint64_t cta_start = cta * PR_T * PR_E;
    if (cta_start >= M) {
        if (t == 0) st(&g_tot[cta], Fq::one());
        return;  // the whole CTA leaves before any barrier
    }
    const uint64_t gt = cta * PR_T + t;
    const uint64_t s64 = cta_start + (uint64_t)t * PR_E;
    uint32_t nj = 0;
    FqL acc = to_l(Fq::one());
    if (s64 < M) {
        const uint32_t s = (uint32_t)s64;
        const uint32_t end = (s64 + PR_E < M) ? s + PR_E : M;
        uint64_t lo = 0, hi = NB;  // in_off[lo] <= s < in_off[hi]
        while (hi - lo > 1) {
            const uint64_t mid = (lo + hi) >> 1;
            if (in_off[mid] <= s) lo = mid; else hi = mid;
        }
        uint64_t b = lo;
        uint32_t bstart = in_off[b], bnext = in_off[b + 1];
        for (uint32_t e = s; e < end; e++) {
            while (e >= bnext) { b++; bstart = bnext; bnext = in_off[b + 1]; }
            const uint32_t local = e - bstart;
            if (local & 1u) continue;
            const uint32_t o = out_off[b] + (local >> 1);
            const G1Affine P1 = pr_load<FIRST>(sorted, src, e);
            if (e + 1 >= bnext) { st_affine(&out_pts[o], P1); continue; }
            const G1Affine P2 = pr_load<FIRST>(sorted, src, e + 1);
            if (is_inf(P1) || is_inf(P2)) { st_affine(&out_pts[o], is_inf(P1) ? P2 : P1); continue; }
            if (P1.x == P2.x && P1.y != P2.y) {  // P2 = -P1
                G1Affine z;
                z.x = Fq::zero(); z.y = Fq::zero();
                st_affine(&out_pts[o], z);
                continue;
            }
            FqL d, num;
            pr_slope_terms(P1, P2, d, num);
            acc = nj == 0 ? d : fl_mul(acc, d);
            st(&g_pref[gt * 4 + nj], from_l(acc));
            g_job[gt * 4 + nj] = make_uint2(e, o);
            nj++;
        }
    }
    g_nj[gt] = nj;
    tree[PR_T + t] = acc;
    __syncthreads();
    for (int w = PR_T / 2; w >= 1; w >>= 1) {
        if (t < w) tree[w + t] = fl_mul(tree[2 * (w + t)], tree[2 * (w + t) + 1]);
        __syncthreads();
    }
    for (int i = t + 1; i < 2 * PR_T; i += PR_T) st(&g_tree[cta * 2 * PR_T + i], from_l(tree[i]));
    if (t == 0) st(&g_tot[cta], from_l(tree[1]));
}

// Backward half: the inverted CTA total (g_tot[cta]) goes down the stored
// tree to every thread, which walks its jobs in reverse, recovers each
// denominator's inverse from its prefix, and writes P1 + P2.
template <bool FIRST>
__global__ void __launch_bounds__(PR_T) k_msm_pair_bwd(const uint32_t* __restrict__ sorted,
                                                       const G1Affine* __restrict__ src,
                                                       const uint32_t* __restrict__ in_off, uint64_t NB,
                                                       G1Affine* __restrict__ out_pts, const Fq* __restrict__ g_pref,
                                                       const uint2* __restrict__ g_job,
                                                       const uint32_t* __restrict__ g_nj,
                                                       const Fq* __restrict__ g_tree, const Fq* __restrict__ g_tot)
{
    __shared__ FqL tree[2 * PR_T];
    const int t = threadIdx.x;
    const uint32_t M = in_off[NB];
    const uint64_t cta = blockIdx.x;
    if (cta * PR_T * PR_E >= M) return;  // the whole CTA
    const uint64_t gt = cta * PR_T + t;
    for (int i = t + 1; i < 2 * PR_T; i += PR_T) tree[i] = to_l(ld(&g_tree[cta * 2 * PR_T + i]));
    __syncthreads();
    if (t == 0) tree[1] = to_l(ld(&g_tot[cta]));
    __syncthreads();
    for (int w = 1; w < PR_T; w <<= 1) {
        if (t < w) {
            const int k = w + t;
            const FqL inv = tree[k], l = tree[2 * k], r = tree[2 * k + 1];
            const Fl2<FqCfg> lr = fl_mul2(inv, r, inv, l);
            tree[2 * k] = lr.a;
            tree[2 * k + 1] = lr.b;
        }
        __syncthreads();
    }
    FqL inv = tree[PR_T + t];
    const int nj = (int)g_nj[gt];
    for (int k = nj - 1; k >= 0; k--) {
        const uint2 job = g_job[gt * 4 + k];
        const G1Affine P1 = pr_load<FIRST>(sorted, src, job.x);
        const G1Affine P2 = pr_load<FIRST>(sorted, src, job.x + 1);
        FqL d, num;
        pr_slope_terms(P1, P2, d, num);
        FqL inv_d;
        if (k > 0) {
            const Fl2<FqCfg> r = fl_mul2(inv, to_l(ld(&g_pref[gt * 4 + k - 1])), inv, d);
            inv_d = r.a;
            inv = r.b;
        } else {
            inv_d = inv;
        }
        const FqL x1 = to_l(P1.x), y1 = to_l(P1.y);
        const FqL lam = fl_mul(num, inv_d);
        const FqL x3 = fl_sub(fl_sub(fl_sqr(lam), x1), to_l(P2.x));
        const FqL y3 = fl_sub(fl_mul(lam, fl_sub(x1, x3)), y1);
        G1Affine R;
        R.x = from_l(x3);
        R.y = from_l(y3);
        st_affine(&out_pts[job.y], R);
    }
}

// Per-bucket entry counts after a pairing round: ceil(count / 2).
__global__ void k_msm_half_counts(const uint32_t* __restrict__ in_off, uint64_t NB, uint32_t* __restrict__ out_cnt)
{
    for (uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; b < NB; b += (uint64_t)gridDim.x * blockDim.x)
        out_cnt[b] = (in_off[b + 1] - in_off[b] + 1) >> 1;
}

#endif  // H2B_EXPERIMENTS

__global__ void k_msm_fixup(const uint32_t* __restrict__ offsets, uint64_t NB, uint32_t K, G1Xyzz* __restrict__ buckets,
                            const G1Xyzz* __restrict__ heads, uint32_t* __restrict__ dense, uint64_t max_dense)
{
    for (uint64_t gb = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; gb < NB; gb += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t s = offsets[gb], e = offsets[gb + 1];
        if (s == e) { st_xyzz(&buckets[gb], xyzz_inf()); continue; }
        uint32_t t0 = s / K, t1 = (e - 1) / K;
        if (t1 == t0) continue;
        if (t1 - t0 > DENSE_LIMIT) {
            uint32_t idx = atomicAdd(&dense[max_dense], 1u);
            if (idx < max_dense) dense[idx] = (uint32_t)gb;
            continue;
        }
        G1XyzzL acc = xyzzl_from(ld_xyzz(&buckets[gb]));
        for (uint32_t t = t0 + 1; t <= t1; t++) xyzzl_add(acc, xyzzl_from(ld_xyzz(&heads[t])));
        st_xyzz(&buckets[gb], xyzzl_to(acc));
    }
}

// CTA-wide tree sum of n XYZZ values produced by get(i); result valid in
// thread 0.  The partial sums stay in 29-bit limb form (latency-oriented
// products: every level of the tree is one dependent addition per thread).
template <class Get>
__device__ G1Xyzz block_sum_xyzz(uint64_t n, Get get)
{
    __shared__ G1XyzzL red[256];
    G1XyzzL acc = xyzzl_inf();
    for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) xyzzl_add(acc, xyzzl_from(get(i)));
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int h = blockDim.x >> 1; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) {
            G1XyzzL a = red[threadIdx.x];
            xyzzl_add(a, red[threadIdx.x + h]);
            red[threadIdx.x] = a;
        }
        __syncthreads();
    }
    G1Xyzz r = xyzzl_to(red[0]);
    __syncthreads();
    return r;
}

// Dense buckets (spanning more than DENSE_LIMIT chunks): DENSE_PIECES CTAs
// each tree-sum a slice of the bucket's chunk partials, then one warp per
// bucket tree-sums the pieces into the bucket.
__global__ void __launch_bounds__(256) k_msm_dense_pieces(const uint32_t* __restrict__ offsets, uint64_t NB,
                                                          uint32_t K, const G1Xyzz* __restrict__ heads,
                                                          const uint32_t* __restrict__ dense,
                                                          G1Xyzz* __restrict__ pieces)
{
    const uint32_t items = dense[NB] * DENSE_PIECES;
    for (uint32_t it = blockIdx.x; it < items; it += gridDim.x) {
        uint32_t i = it / DENSE_PIECES, p = it % DENSE_PIECES;
        uint32_t gb = dense[i];
        uint32_t t0 = offsets[gb] / K, t1 = (offsets[gb + 1] - 1) / K;
        uint64_t len = t1 - t0;  // heads t0+1 .. t1
        uint64_t b0 = len * p / DENSE_PIECES, b1 = len * (p + 1) / DENSE_PIECES;
        G1Xyzz r = block_sum_xyzz(b1 - b0, [&](uint64_t j) { return ld_xyzz(&heads[t0 + 1 + b0 + j]); });
        if (threadIdx.x == 0) st_xyzz(&pieces[it], r);
        __syncthreads();
    }
}

__global__ void __launch_bounds__(DENSE_PIECES) k_msm_dense_merge(const uint64_t NB, G1Xyzz* __restrict__ buckets,
                                                                  const uint32_t* __restrict__ dense,
                                                                  const G1Xyzz* __restrict__ pieces)
{
    __shared__ G1Xyzz red[DENSE_PIECES];
    const uint32_t cnt = dense[NB];
    for (uint32_t i = blockIdx.x; i < cnt; i += gridDim.x) {
        red[threadIdx.x] = ld_xyzz(&pieces[(uint64_t)i * DENSE_PIECES + threadIdx.x]);
        __syncthreads();
        for (int h = DENSE_PIECES / 2; h > 0; h >>= 1) {
            if ((int)threadIdx.x < h) {
                G1Xyzz a = red[threadIdx.x];
                xyzz_add(a, red[threadIdx.x + h]);
                red[threadIdx.x] = a;
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            uint32_t gb = dense[i];
            G1Xyzz acc = ld_xyzz(&buckets[gb]);
            xyzz_add(acc, red[0]);
            st_xyzz(&buckets[gb], acc);
        }
        __syncthreads();
    }
}

// Bucket reduction, W_w = sum_{j<H} (j+1) B_{w,j}, in three parallel steps.
// 1. Thread (w, s), segment s = buckets s*L .. s*L+L-1:
//      acc_s = sum_j (j - sL + 1) B_j      run_s = sum_j B_j
// 2. CTA (w, k): k < NBITS: T_k = sum over s with bit k set of run_s;
//                k = NBITS: T = sum_s acc_s.
// 3. Thread w: W_w = T + L * sum_k 2^k T_k (Horner over the bits).
__global__ void __launch_bounds__(128) k_msm_segments(const G1Xyzz* __restrict__ buckets, int W, uint32_t H,
                                                      uint32_t L, uint32_t S, G1Xyzz* __restrict__ segacc,
                                                      G1Xyzz* __restrict__ segrun)
{
    uint64_t total = (uint64_t)W * S;
    for (uint64_t id = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; id < total;
         id += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t w = id / S, s = id % S;
        const G1Xyzz* B = buckets + w * H + s * L;
        G1XyzzL run = xyzzl_inf(), acc = xyzzl_inf();
        for (int j = (int)L - 1; j >= 0; j--) {
            xyzzl_add(run, xyzzl_from(ld_xyzz(&B[j])));
            xyzzl_add(acc, run);
        }
        st_xyzz(&segacc[id], xyzzl_to(acc));
        st_xyzz(&segrun[id], xyzzl_to(run));
    }
}

// CTA (w, k, part): part `part` of BP of bit sum (w, k); with BP = 1 the
// CTA writes the bit sum itself, else its partial (out[(w, k) * BP + part]).
__global__ void __launch_bounds__(256) k_msm_bitsums(const G1Xyzz* __restrict__ segacc,
                                                     const G1Xyzz* __restrict__ segrun, uint32_t S, int nbits,
                                                     uint32_t BP, G1Xyzz* __restrict__ out)
{
    const uint32_t wk = blockIdx.x / BP, part = blockIdx.x % BP;
    const uint32_t w = wk / (nbits + 1);
    const int k = (int)(wk % (nbits + 1));
    // k == nbits: all S weighted sums; else the S/2 plain sums with bit k set,
    // s = (hi << (k+1)) | (1 << k) | lo
    const bool all = (k == nbits);
    const uint64_t lo_mask = all ? 0 : (1ull << k) - 1;
    const uint64_t items = all ? S : S / 2;
    const uint64_t per = (items + BP - 1) / BP;
    const uint64_t j0 = std::min<uint64_t>(items, (uint64_t)part * per);
    const uint64_t j1 = std::min<uint64_t>(items, j0 + per);
    G1Xyzz r = block_sum_xyzz(j1 - j0, [&](uint64_t jj) {
        const uint64_t j = j0 + jj;
        if (all) return ld_xyzz(&segacc[(uint64_t)w * S + j]);
        uint64_t s = ((j & ~lo_mask) << 1) | (1ull << k) | (j & lo_mask);
        return ld_xyzz(&segrun[(uint64_t)w * S + s]);
    });
    if (threadIdx.x == 0) st_xyzz(&out[blockIdx.x], r);
}

// CTA (w, k): the BP partials of bit sum (w, k).
__global__ void __launch_bounds__(256) k_msm_bitparts(const G1Xyzz* __restrict__ parts, uint32_t BP,
                                                      G1Xyzz* __restrict__ bits)
{
    G1Xyzz r = block_sum_xyzz(BP, [&](uint64_t j) { return ld_xyzz(&parts[(uint64_t)blockIdx.x * BP + j]); });
    if (threadIdx.x == 0) st_xyzz(&bits[blockIdx.x], r);
}

// One warp per window (warps loop when there are more windows than warps in
// the grid), the Horner steps on the lane-parallel formulas.
__global__ void k_msm_wincombine(const G1Xyzz* __restrict__ bits, int W, int nbits, int log_l,
                                 G1Xyzz* __restrict__ wins)
{
    const int warps = (int)(gridDim.x * (blockDim.x >> 5));
    for (int w = (int)(blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)); w < W; w += warps) {
        const G1Xyzz* T = bits + (uint64_t)w * (nbits + 1);
        G1XyzzL r = xyzzl_inf();
        for (int k = nbits - 1; k >= 0; k--) {
            r = xyzzw_dbl(r);
            xyzzw_add(r, xyzzl_from(ld_xyzz(&T[k])));
        }
        for (int d = 0; d < log_l; d++) r = xyzzw_dbl(r);
        xyzzw_add(r, xyzzl_from(ld_xyzz(&T[nbits])));
        if ((threadIdx.x & 31) == 0) st_xyzz(&wins[w], xyzzl_to(r));
    }
}

// 2^(c*w) * W_w with one warp per window (lane-parallel doublings), then the
// sum over windows and the affine conversion by the first warp.
constexpr int FINAL_MAX_W = 64;
__global__ void k_msm_final(const G1Xyzz* __restrict__ wins, int W, int c, G1Jac* __restrict__ out)
{
    __shared__ G1Xyzz sh[FINAL_MAX_W];
    for (int w = (int)(threadIdx.x >> 5); w < W; w += (int)(blockDim.x >> 5)) {
        G1XyzzL x = xyzzl_from(ld_xyzz(&wins[w]));
        for (int d = 0; d < c * w; d++) x = xyzzw_dbl(x);
        if ((threadIdx.x & 31) == 0) sh[w] = xyzzl_to(x);
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        G1XyzzL acc = xyzzl_inf();
        for (int i = 0; i < W; i++) xyzzw_add(acc, xyzzl_from(sh[i]));
        if (threadIdx.x == 0) {
            G1Jac j = xyzz_to_jac_affine(xyzzl_to(acc));
            st(&out->X, j.X);
            st(&out->Y, j.Y);
            st(&out->Z, j.Z);
        }
    }
}

__global__ void k_write_inf(G1Jac* out)
{
    if (threadIdx.x == 0) {
        st(&out->X, Fq::zero());
        st(&out->Y, Fq::one());
        st(&out->Z, Fq::zero());
    }
}

// A merged run over a window table: window j of the reduction is job j's
// whole sum (the table already holds the window multiples), so each job's
// result is its window sum in the reference's affine image, one lane per job.
struct MsmOuts {
    G1Jac* p[MSM_MERGE_MAX];
};
__global__ void k_msm_final_each(const G1Xyzz* __restrict__ wins, uint32_t J, const __grid_constant__ MsmOuts outs)
{
    const uint32_t j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (j >= J || (threadIdx.x & 31) != 0) return;
    const G1Jac r = xyzz_to_jac_affine(ld_xyzz(&wins[j]));
    st(&outs.p[j]->X, r.X);
    st(&outs.p[j]->Y, r.Y);
    st(&outs.p[j]->Z, r.Z);
}

// Per-bit sums of the segment sums (reduction step 2), in BP parts per sum
// when the segments are many.
static RustError msm_bitsums(const MsmPlan& p, const MsmScratch& s, cudaStream_t st)
{
    const uint32_t nbs = (uint32_t)p.Wr * (uint32_t)(p.NBITS + 1);
    k_msm_bitsums<<<nbs * p.BP, 256, 0, st>>>(s.segacc, s.segrun, p.S, p.NBITS, p.BP, p.BP > 1 ? s.bitparts : s.bits);
    H2B_LAUNCHED("k_msm_bitsums");
    if (p.BP > 1) {
        k_msm_bitparts<<<nbs, 256, 0, st>>>(s.bitparts, p.BP, s.bits);
        H2B_LAUNCHED("k_msm_bitparts");
    }
    return ok();
}

// Runs steps 1-7 on device buffers; result (96 bytes) lands in s.result.
// The lazy accumulation (window tables are stored in its form; plain bases
// are converted by the split kernel) unless pairing rounds or an older
// variant run.
static bool msm_lazy(const MsmPlan& p)
{
    return p.R == 0 && (p.tn > 0 || g_msm_acc_variant == 0 || g_msm_acc_variant >= 6);
}

// Phases of one MSM on `st`: msm_begin clears the histogram, msm_split takes
// points [lo, hi) through the GLV split (and base conversion) and the
// histogram -- callers may feed the points in pieces as they arrive --, and
// msm_finish sorts, accumulates and reduces.
static RustError msm_begin(const MsmPlan& p, const MsmScratch& s, cudaStream_t st)
{
    prof_begin(PROF_MSM_TOTAL, st);
    H2B_CUDA(cudaMemsetAsync(s.counts, 0, p.NB * sizeof(uint32_t), st));
    H2B_CUDA(cudaMemsetAsync(s.dense + p.max_dense, 0, sizeof(uint32_t), st));
    return ok();
}

static RustError msm_split(const MsmPlan& p, const MsmScratch& s, const Fr* d_scalars, const G1Affine* d_bases,
                           uint64_t lo, uint64_t hi, cudaStream_t st)
{
    if (hi <= lo) return ok();
    const unsigned sm_cap = 148u * 16u;
    uint4* vsc = reinterpret_cast<uint4*>(s.canon);  // 2n x 16 B in the n x 32 B slot
    k_msm_glv_hist<<<grid_for(hi - lo, 256, sm_cap), 256, 0, st>>>(
        d_scalars, vsc, lo, hi, d_bases, msm_lazy(p) && p.tn == 0 ? s.rbases : nullptr, p.n, p.c, p.W, p.H, s.counts,
        p.tn);
    H2B_LAUNCHED("k_msm_glv_hist");
    return ok();
}

static RustError msm_finish(const MsmPlan& p, const MsmScratch& s, const G1Affine* d_bases, cudaStream_t st)
{
    const unsigned sm_cap = 148u * 16u;
    const uint4* vsc = reinterpret_cast<const uint4*>(s.canon);
    const bool lazy = msm_lazy(p);
    H2B_CUDA(scan_u32(s.counts, p.NB, s.offsets, s.scan_tmp, st));
    H2B_CUDA(cudaMemcpyAsync(s.cursor, s.offsets, p.NB * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    k_msm_sort<true><<<grid_for(p.nv, 256, sm_cap), 256, 0, st>>>(vsc, 0, p.nv, p.c, p.W, p.H, s.cursor,
                                                                    s.sorted, p.tn, 0u);
    H2B_LAUNCHED("k_msm_sort<scatter>");
    prof_begin(PROF_MSM_ACCUMULATE, st);
    // pairing rounds: sorted entries -> pts[0] -> pts[1] -> pts[0]
    const uint32_t* off = s.offsets;
#if H2B_EXPERIMENTS
    const G1Affine* src = d_bases;
    for (int r = 1; r <= p.R; r++) {
        k_msm_half_counts<<<grid_for(p.NB, 256, sm_cap), 256, 0, st>>>(off, p.NB, s.counts);
        H2B_LAUNCHED("k_msm_half_counts");
        H2B_CUDA(scan_u32(s.counts, p.NB, s.roff[r - 1], s.scan_tmp, st));
        G1Affine* dst = s.pts[(r - 1) & 1];
        const uint64_t ctas = pr_ctas(p.cap[r - 1]);
        const uint32_t* srt = r == 1 ? s.sorted : nullptr;
        if (r == 1)
            k_msm_pair_fwd<true><<<(unsigned)ctas, PR_T, 0, st>>>(srt, src, off, p.NB, s.roff[0], dst, s.pr_pref,
                                                                  s.pr_job, s.pr_nj, s.pr_tree, s.pr_tot);
        else
            k_msm_pair_fwd<false><<<(unsigned)ctas, PR_T, 0, st>>>(srt, src, off, p.NB, s.roff[r - 1], dst,
                                                                   s.pr_pref, s.pr_job, s.pr_nj, s.pr_tree, s.pr_tot);
        H2B_LAUNCHED("k_msm_pair_fwd");
        H2B_TRY(fq_batch_invert(s.pr_tot, ctas, s.pr_inv_scratch, s.pr_inv_bytes, st));
        if (r == 1)
            k_msm_pair_bwd<true><<<(unsigned)ctas, PR_T, 0, st>>>(srt, src, off, p.NB, dst, s.pr_pref, s.pr_job,
                                                                  s.pr_nj, s.pr_tree, s.pr_tot);
        else
            k_msm_pair_bwd<false><<<(unsigned)ctas, PR_T, 0, st>>>(srt, src, off, p.NB, dst, s.pr_pref, s.pr_job,
                                                                   s.pr_nj, s.pr_tree, s.pr_tot);
        H2B_LAUNCHED("k_msm_pair_bwd");
        off = s.roff[r - 1];
        src = dst;
    }
#endif
    const uint64_t chunks = (p.cap[p.R] + p.Kf - 1) / p.Kf;
    const unsigned acc_grid = grid_for(chunks, 128, 148u * 32u);
    if (lazy && g_msm_acc_variant == 6)
        k_msm_accumulate_d<<<acc_grid, 128, 0, st>>>(s.sorted, off, p.NB, p.Kf, p.tn ? d_bases : s.rbases,
                                                     p.tn ? (uint64_t)p.W * p.tn : p.n, s.buckets, s.heads,
                                                     g_msm_prefetch);
#if H2B_EXPERIMENTS
    else if (lazy && g_msm_acc_variant == 7)
        k_msm_accumulate_d2<<<acc_grid, 128, 0, st>>>(s.sorted, off, p.NB, p.Kf, p.tn ? d_bases : s.rbases,
                                                      p.tn ? (uint64_t)p.W * p.tn : p.n, s.buckets, s.heads);
#endif
    else if (lazy)
        k_msm_accumulate_z<<<acc_grid, 128, 0, st>>>(s.sorted, off, p.NB, p.Kf, p.tn ? d_bases : s.rbases,
                                                     p.tn ? (uint64_t)p.W * p.tn : p.n, s.buckets, s.heads);
#if H2B_EXPERIMENTS
    else if (p.R > 0)
        k_msm_accumulate<2, true><<<acc_grid, 128, 0, st>>>(nullptr, off, p.NB, p.Kf, src, s.buckets, s.heads);
    else if (g_msm_acc_variant == 5)
        k_msm_accumulate<0, false><<<acc_grid, 128, 0, st>>>(s.sorted, off, p.NB, p.Kf, src, s.buckets, s.heads);
    else if (g_msm_acc_variant == 1)
        k_msm_accumulate<1, false><<<acc_grid, 128, 0, st>>>(s.sorted, off, p.NB, p.Kf, src, s.buckets, s.heads);
    else if (g_msm_acc_variant == 2)
        k_msm_accumulate<2, false><<<acc_grid, 128, 0, st>>>(s.sorted, off, p.NB, p.Kf, src, s.buckets, s.heads);
    else if (g_msm_acc_variant == 3)
        k_msm_accumulate<3, false><<<acc_grid, 128, 0, st>>>(s.sorted, off, p.NB, p.Kf, src, s.buckets, s.heads);
    else if (g_msm_acc_variant == 4)
        k_msm_accumulate<4, false><<<acc_grid, 128, 0, st>>>(s.sorted, off, p.NB, p.Kf, src, s.buckets, s.heads);
#endif
    prof_end(PROF_MSM_ACCUMULATE, st);
    H2B_LAUNCHED("k_msm_accumulate");
    k_msm_fixup<<<grid_for(p.NB, 128, sm_cap), 128, 0, st>>>(off, p.NB, p.Kf, s.buckets, s.heads, s.dense,
                                                            p.max_dense);
    H2B_LAUNCHED("k_msm_fixup");
    k_msm_dense_pieces<<<148 * 4, 256, 0, st>>>(off, p.max_dense, p.Kf, s.heads, s.dense, s.pieces);
    H2B_LAUNCHED("k_msm_dense_pieces");
    k_msm_dense_merge<<<148, DENSE_PIECES, 0, st>>>(p.max_dense, s.buckets, s.dense, s.pieces);
    H2B_LAUNCHED("k_msm_dense_merge");
    uint64_t nseg = (uint64_t)p.Wr * p.S;
    k_msm_segments<<<grid_for(nseg, 128, sm_cap), 128, 0, st>>>(s.buckets, p.Wr, p.H, p.L, p.S, s.segacc, s.segrun);
    H2B_LAUNCHED("k_msm_segments");
    H2B_TRY(msm_bitsums(p, s, st));
    k_msm_wincombine<<<(p.Wr + 7) / 8, 32 * std::min(p.Wr, 8), 0, st>>>(s.bits, p.Wr, p.NBITS, p.LOGL, s.wins);
    H2B_LAUNCHED("k_msm_wincombine");
    k_msm_final<<<1, 32 * std::min(p.Wr, 8), 0, st>>>(s.wins, p.Wr, p.c, s.result);
    prof_end(PROF_MSM_TOTAL, st);
    H2B_LAUNCHED("k_msm_final");
    return ok();
}

RustError msm_run(const MsmPlan& p, const MsmScratch& s, const Fr* d_scalars, const G1Affine* d_bases, cudaStream_t st)
{
    if (p.n == 0) {
        k_write_inf<<<1, 32, 0, st>>>(s.result);
        H2B_LAUNCHED("k_write_inf");
        return ok();
    }
    H2B_TRY(msm_begin(p, s, st));
    H2B_TRY(msm_split(p, s, d_scalars, d_bases, 0, p.n, st));
    return msm_finish(p, s, d_bases, st);
}

RustError msm_run_merged(const MsmPlan& p, const MsmScratch& s, uint32_t J, const Fr* const* scalars,
                         const uint64_t* ns, const G1Affine* table, G1Jac* const* outs, cudaStream_t st)
{
    if (J == 0) return ok();
    if (J > (uint32_t)MSM_MERGE_MAX || p.tn == 0 || (uint32_t)p.Wr != J)
        return err(cudaErrorInvalidValue, "msm_run_merged: plan does not match the jobs");
    const unsigned sm_cap = 148u * 16u;
    uint4* vsc = reinterpret_cast<uint4*>(s.canon);
    prof_begin(PROF_MSM_TOTAL, st);
    H2B_CUDA(cudaMemsetAsync(s.counts, 0, p.NB * sizeof(uint32_t), st));
    H2B_CUDA(cudaMemsetAsync(s.dense + p.max_dense, 0, sizeof(uint32_t), st));
    uint64_t at = 0;   // job j's virtual scalars start at vsc + 2 * at
    for (uint32_t j = 0; j < J; j++) {
        if (ns[j] == 0) continue;
        k_msm_glv<<<grid_for(ns[j], 256, sm_cap), 256, 0, st>>>(scalars[j], vsc + 2 * at, 0, ns[j], nullptr, nullptr,
                                                                ns[j]);
        H2B_LAUNCHED("k_msm_glv");
        k_msm_sort<false><<<grid_for(2 * ns[j], 256, sm_cap), 256, 0, st>>>(vsc + 2 * at, 0, 2 * ns[j], p.c, p.W,
                                                                              p.H, s.counts, nullptr, p.tn, j * p.H);
        H2B_LAUNCHED("k_msm_sort<hist>");
        at += ns[j];
    }
    H2B_CUDA(scan_u32(s.counts, p.NB, s.offsets, s.scan_tmp, st));
    H2B_CUDA(cudaMemcpyAsync(s.cursor, s.offsets, p.NB * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    at = 0;
    for (uint32_t j = 0; j < J; j++) {
        if (ns[j] == 0) continue;
        k_msm_sort<true><<<grid_for(2 * ns[j], 256, sm_cap), 256, 0, st>>>(vsc + 2 * at, 0, 2 * ns[j], p.c, p.W, p.H,
                                                                             s.cursor, s.sorted, p.tn, j * p.H);
        H2B_LAUNCHED("k_msm_sort<scatter>");
        at += ns[j];
    }
    prof_begin(PROF_MSM_ACCUMULATE, st);
    const uint64_t chunks = (p.max_entries + p.Kf - 1) / p.Kf;
    const unsigned acc_grid = grid_for(chunks, 128, 148u * 32u);
    if (g_msm_acc_variant == 6)
        k_msm_accumulate_d<<<acc_grid, 128, 0, st>>>(s.sorted, s.offsets, p.NB, p.Kf, table, (uint64_t)p.W * p.tn,
                                                     s.buckets, s.heads, g_msm_prefetch);
    else
        k_msm_accumulate_z<<<acc_grid, 128, 0, st>>>(s.sorted, s.offsets, p.NB, p.Kf, table, (uint64_t)p.W * p.tn,
                                                     s.buckets, s.heads);
    prof_end(PROF_MSM_ACCUMULATE, st);
    H2B_LAUNCHED("k_msm_accumulate");
    k_msm_fixup<<<grid_for(p.NB, 128, sm_cap), 128, 0, st>>>(s.offsets, p.NB, p.Kf, s.buckets, s.heads, s.dense,
                                                            p.max_dense);
    H2B_LAUNCHED("k_msm_fixup");
    k_msm_dense_pieces<<<148 * 4, 256, 0, st>>>(s.offsets, p.max_dense, p.Kf, s.heads, s.dense, s.pieces);
    H2B_LAUNCHED("k_msm_dense_pieces");
    k_msm_dense_merge<<<148, DENSE_PIECES, 0, st>>>(p.max_dense, s.buckets, s.dense, s.pieces);
    H2B_LAUNCHED("k_msm_dense_merge");
    const uint64_t nseg = (uint64_t)p.Wr * p.S;
    k_msm_segments<<<grid_for(nseg, 128, sm_cap), 128, 0, st>>>(s.buckets, p.Wr, p.H, p.L, p.S, s.segacc, s.segrun);
    H2B_LAUNCHED("k_msm_segments");
    H2B_TRY(msm_bitsums(p, s, st));
    k_msm_wincombine<<<(p.Wr + 7) / 8, 32 * std::min(p.Wr, 8), 0, st>>>(s.bits, p.Wr, p.NBITS, p.LOGL, s.wins);
    H2B_LAUNCHED("k_msm_wincombine");
    MsmOuts o;
    for (uint32_t j = 0; j < J; j++) o.p[j] = outs[j];
    k_msm_final_each<<<(J + 7) / 8, 256, 0, st>>>(s.wins, J, o);
    prof_end(PROF_MSM_TOTAL, st);
    H2B_LAUNCHED("k_msm_final_each");
    return ok();
}

} // namespace h2b

using namespace h2b;

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

static uint64_t msm_ws(uint64_t length, bool scalar_host, bool bases_host)
{
    MsmPlan p = msm_plan(length);
    ScratchPlan sp;
    msm_plan_scratch(p, sp, scalar_host, bases_host);
    return sp.used;
}

extern "C" uint64_t _halo2_msm_max_length(uint64_t free_bytes)
{
    for (int lg = 27; lg > 0; lg--) {
        if (msm_ws(1ull << lg, true, true) < free_bytes) return 1ull << lg;
    }
    return 0;
}

extern "C" uint64_t _halo2_multiexp_workspace_size(uint64_t length) { return msm_ws(length, true, true); }
extern "C" uint64_t _halo2_multiexp_device_bases_workspace_size(uint64_t length) { return msm_ws(length, true, false); }
extern "C" uint64_t _halo2_multiexp_device_scalars_device_bases_workspace_size(uint64_t length)
{
    return msm_ws(length, false, false);
}

static RustError msm_entry(const void* scalars, bool scalar_host, const void* bases, bool bases_host, void* h_out,
                           uint64_t length, void* scratch, uint64_t scratch_bytes, cudaStream_t st, const char* who)
{
    if (length > MSM_MAX_LENGTH) return err(cudaErrorInvalidValue, "MSM length above 2^27 points");
    MsmPlan p = msm_plan(length);
    uint64_t need = msm_ws(length, scalar_host, bases_host);
    if (scratch_bytes < need) return scratch_too_small(who, scratch_bytes, need);
    ScratchArena ar(scratch, scratch_bytes);
    MsmScratch s = msm_carve(p, ar, scalar_host, bases_host);
    if (!ar.good()) return scratch_too_small(who, scratch_bytes, need);
    const Fr* d_sc = (const Fr*)scalars;
    const G1Affine* d_b = (const G1Affine*)bases;
    if (length > 0 && bases_host) {
        H2B_CUDA(cudaMemcpyAsync(s.bases_stage, bases, length * sizeof(G1Affine), cudaMemcpyHostToDevice, st));
        d_b = s.bases_stage;
    }
    if (length >= MSM_PIPE_MIN && scalar_host) {
        // Host scalars arrive in MSM_PIPE_PIECES pieces on a forked copy stream;
        // the split and histogram of each piece run while the next one copies.
        cudaStream_t cs;
        H2B_TRY(h2b_exec_fork(st, 1, &cs));
        cudaEvent_t ev[MSM_PIPE_PIECES];
        for (int i = 0; i < MSM_PIPE_PIECES; i++) H2B_CUDA(cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming));
        RustError e = msm_begin(p, s, st);
        for (int i = 0; i < MSM_PIPE_PIECES && e.code == 0; i++) {
            const uint64_t lo = length * i / MSM_PIPE_PIECES, hi = length * (i + 1) / MSM_PIPE_PIECES;
            cudaError_t c = cudaMemcpyAsync(s.scalar_stage + lo, (const Fr*)scalars + lo, (hi - lo) * sizeof(Fr),
                                            cudaMemcpyHostToDevice, cs);
            if (c == cudaSuccess) c = cudaEventRecord(ev[i], cs);
            if (c == cudaSuccess) c = cudaStreamWaitEvent(st, ev[i], 0);
            e = c == cudaSuccess ? msm_split(p, s, s.scalar_stage, d_b, lo, hi, st) : cuda_err(c, who);
        }
        for (int i = 0; i < MSM_PIPE_PIECES; i++) cudaEventDestroy(ev[i]);
        H2B_TRY(e);
        H2B_TRY(msm_finish(p, s, d_b, st));
    } else {
        if (length > 0 && scalar_host) {
            H2B_CUDA(cudaMemcpyAsync(s.scalar_stage, scalars, length * sizeof(Fr), cudaMemcpyHostToDevice, st));
            d_sc = s.scalar_stage;
        }
        H2B_TRY(msm_run(p, s, d_sc, d_b, st));
    }
    H2B_CUDA(cudaMemcpyAsync(h_out, s.result, sizeof(G1Jac), cudaMemcpyDeviceToHost, st));
    H2B_CUDA(cudaStreamSynchronize(st));
    return ok();
}

extern "C" RustError _halo2_multiexp(const FFITraitObject* scalar, const FFITraitObject* point,
                                     const FFITraitObject* output, uint64_t length, void* scratch,
                                     uint64_t scratch_bytes, cudaStream_t stream)
{
    return msm_entry(scalar->ptr, true, point->ptr, true, output->ptr, length, scratch, scratch_bytes, stream,
                     "_halo2_multiexp");
}

extern "C" RustError _halo2_multiexp_device_bases(const FFITraitObject* h_scalar, const void* d_bases,
                                                  const FFITraitObject* h_output, uint64_t length, void* scratch,
                                                  uint64_t scratch_bytes, cudaStream_t stream)
{
    return msm_entry(h_scalar->ptr, true, d_bases, false, h_output->ptr, length, scratch, scratch_bytes, stream,
                     "_halo2_multiexp_device_bases");
}

extern "C" RustError _halo2_multiexp_device_scalars_device_bases(const void* d_scalar, const void* d_bases,
                                                                 const FFITraitObject* h_output, uint64_t length,
                                                                 void* scratch, uint64_t scratch_bytes,
                                                                 cudaStream_t stream)
{
    return msm_entry(d_scalar, false, d_bases, false, h_output->ptr, length, scratch, scratch_bytes, stream,
                     "_halo2_multiexp_device_scalars_device_bases");
}

// Device-output, sync-free variant: the 96-byte Jacobian image is written to
// d_out on `stream`.  Same scratch size as the device-scalars entry point.
extern "C" RustError h2b_msm_device(const void* d_scalar, const void* d_bases, void* d_out, uint64_t length,
                                    void* scratch, uint64_t scratch_bytes, cudaStream_t stream)
{
    if (length > MSM_MAX_LENGTH) return err(cudaErrorInvalidValue, "MSM length above 2^27 points");
    MsmPlan p = msm_plan(length);
    uint64_t need = msm_ws(length, false, false);
    if (scratch_bytes < need) return scratch_too_small("h2b_msm_device", scratch_bytes, need);
    ScratchArena ar(scratch, scratch_bytes);
    MsmScratch s = msm_carve(p, ar, false, false);
    H2B_TRY(msm_run(p, s, (const Fr*)d_scalar, (const G1Affine*)d_bases, stream));
    H2B_CUDA(cudaMemcpyAsync(d_out, s.result, sizeof(G1Jac), cudaMemcpyDeviceToDevice, stream));
    return ok();
}

// ---- precomputed window tables (SRS kept resident with its window multiples) --
// A table for n bases holds W slices of n affine points, slice w being
// [2^(c w)] P_i (c and W from the n-point plan).  An MSM over the table puts
// the digits of every window into one bucket set, so the bucket reduction
// covers one window and the final 2^(c w) doubling chain disappears; the
// entry count (bucket additions) is unchanged.  Slice w + 1 is c doublings of
// slice w, made affine with one batch inversion per slice.

namespace h2b {

__global__ void k_table_double(const G1Affine* __restrict__ prev, uint64_t n, int c, G1Xyzz* __restrict__ tmp,
                               Fq* __restrict__ den)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const G1Affine P = ld_affine(&prev[i]);
        if (is_inf(P)) {
            st_xyzz(&tmp[i], xyzz_inf());
            st(&den[i], Fq::zero());
            continue;
        }
        G1Xyzz X = xyzz_dbl_affine(P);
        for (int k = 1; k < c; k++) X = xyzz_dbl(X);
        st_xyzz(&tmp[i], X);
        st(&den[i], X.ZZ * X.ZZZ);
    }
}

// den_inv[i] = 1 / (ZZ ZZZ): x = X ZZZ / (ZZ ZZZ), y = Y ZZ / (ZZ ZZZ); zero -> infinity (0, 0).
__global__ void k_table_affine(const G1Xyzz* __restrict__ tmp, const Fq* __restrict__ den_inv, uint64_t n,
                               G1Affine* __restrict__ out)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const Fq d = ld(&den_inv[i]);
        G1Affine a;
        if (d.is_zero()) {
            a.x = Fq::zero();
            a.y = Fq::zero();
        } else {
            const G1Xyzz X = ld_xyzz(&tmp[i]);
            a.x = X.X * (d * X.ZZZ);
            a.y = X.Y * (d * X.ZZ);
        }
        st(&out[i].x, a.x);
        st(&out[i].y, a.y);
    }
}

// Layout of a window table for tn bases: the untuned window width, which
// msm_plan_table also uses, so tuning never changes a table's meaning.
static MsmPlan table_layout_plan(uint64_t tn) { return plan_core(tn, choose_c(tn), 0); }

// Entries encode the table point as 2 (w tn + i) + half in 31 bits.
static bool table_fits(uint64_t tn)
{
    const MsmPlan p = table_layout_plan(tn);
    return tn > 0 && tn <= MSM_MAX_LENGTH && 2 * (uint64_t)p.W * tn < (1ull << 31);
}

} // namespace h2b

// W window slices of n points, then the same W slices under phi (x -> beta x).
extern "C" uint64_t h2b_msm_table_points(uint64_t n)
{
    if (!table_fits(n)) return 0;
    return 2 * (uint64_t)table_layout_plan(n).W * n;
}

extern "C" uint64_t h2b_msm_table_precompute_workspace_size(uint64_t n)
{
    if (!table_fits(n)) return 0;
    ScratchPlan sp;
    sp.add_n<G1Xyzz>(n);
    sp.add_n<Fq>(n);
    sp.add(fq_batch_invert_scratch(n));
    return sp.used;
}

// d_table receives h2b_msm_table_points(n) affine points; d_bases is not modified.
extern "C" RustError h2b_msm_table_precompute(const void* d_bases, uint64_t n, void* d_table, void* scratch,
                                              uint64_t scratch_bytes, cudaStream_t stream)
{
    if (!table_fits(n)) return err(cudaErrorInvalidValue, "h2b_msm_table_precompute: n out of range");
    const MsmPlan p = table_layout_plan(n);
    ScratchArena ar(scratch, scratch_bytes);
    G1Xyzz* tmp = ar.take_n<G1Xyzz>(n);
    Fq* den = ar.take_n<Fq>(n);
    const uint64_t inv_bytes = fq_batch_invert_scratch(n);
    void* inv_scratch = ar.take(inv_bytes);
    if (!ar.good())
        return scratch_too_small("h2b_msm_table_precompute", scratch_bytes, h2b_msm_table_precompute_workspace_size(n));
    G1Affine* table = (G1Affine*)d_table;
    H2B_CUDA(cudaMemcpyAsync(table, d_bases, n * sizeof(G1Affine), cudaMemcpyDeviceToDevice, stream));
    for (int w = 1; w < p.W; w++) {
        k_table_double<<<grid_for(n, 128, 148u * 16u), 128, 0, stream>>>(table + (uint64_t)(w - 1) * n, n, p.c, tmp,
                                                                         den);
        H2B_LAUNCHED("k_table_double");
        H2B_TRY(fq_batch_invert(den, n, inv_scratch, inv_bytes, stream));
        k_table_affine<<<grid_for(n, 256), 256, 0, stream>>>(tmp, den, n, table + (uint64_t)w * n);
        H2B_LAUNCHED("k_table_affine");
    }
    // the accumulation reads the table in the lazy x 2^261 form, with the
    // phi images of all slices after them
    const uint64_t pts = (uint64_t)p.W * n;
    k_to_r261<<<grid_for(pts, 256, 148u * 8u), 256, 0, stream>>>(table, table, pts, table + pts);
    H2B_LAUNCHED("k_to_r261");
    return ok();
}

extern "C" uint64_t h2b_msm_table_workspace_size(uint64_t n, uint64_t table_n)
{
    if (n > table_n || !table_fits(table_n)) return 0;
    const MsmPlan p = msm_plan_table(n, table_n);
    ScratchPlan sp;
    msm_plan_scratch(p, sp, false, false);
    return sp.used;
}

// MSM of n <= table_n device scalars over a table built for table_n bases
// (its first n points of every slice are used); result to d_out (96 B, device).
extern "C" RustError h2b_msm_device_table(const void* d_scalars, const void* d_table, uint64_t table_n, void* d_out,
                                          uint64_t n, void* scratch, uint64_t scratch_bytes, cudaStream_t stream)
{
    if (n > table_n || !table_fits(table_n))
        return err(cudaErrorInvalidValue, "h2b_msm_device_table: n above the table size, or table size out of range");
    const MsmPlan p = msm_plan_table(n, table_n);
    const uint64_t need = h2b_msm_table_workspace_size(n, table_n);
    if (scratch_bytes < need) return scratch_too_small("h2b_msm_device_table", scratch_bytes, need);
    ScratchArena ar(scratch, scratch_bytes);
    MsmScratch s = msm_carve(p, ar, false, false);
    H2B_TRY(msm_run(p, s, (const Fr*)d_scalars, (const G1Affine*)d_table, stream));
    H2B_CUDA(cudaMemcpyAsync(d_out, s.result, sizeof(G1Jac), cudaMemcpyDeviceToDevice, stream));
    return ok();
}

extern "C" void h2b_msm_set_tuning(int window_bits, int chunk) { msm_set_tuning(window_bits, chunk); }

// Form and call structure of the bucket-accumulation kernel: 6 = the lazy
// R' = 2^260 form on the FP64 pipe (default; window tables use it too);
// 0 = the lazy R = 2^261 form of 29-bit limbs with one-step carries on the
// integer multiply pipe (window tables use it for every choice but 6).
// Built with H2B_EXPERIMENTS=1 only, the normalised R = 2^256 limb form with
// 5 = two products per out-of-line call, 1 = all products inline, 2 = one
// product per call, 3 and 4 = one product per call with at most 128 / 96
// registers, and 7 = the FP64 lazy form with two accumulation chains per
// thread (25.7 ms at 2^22).  Measured at 2^22 with the witness-like scalar mix: 6 takes
// 12.26 ms, 0 13.56 ms.  Results are identical; only speed differs.  A value
// that is not built leaves the setting unchanged (read it back with
// h2b_msm_get_accumulate_variant).
extern "C" void h2b_msm_set_accumulate_variant(int v)
{
    if (v == 0 || v == 6 || (H2B_EXPERIMENTS && v >= 1 && v <= 7)) g_msm_acc_variant = v;
}

extern "C" int h2b_msm_get_accumulate_variant(void) { return g_msm_acc_variant; }

// Distance (sorted entries ahead, 0..64) at which the FP64 accumulation
// prefetches the next points into L2; 0 turns it off.  Same results.
extern "C" void h2b_msm_set_prefetch(int distance)
{
    if (distance >= 0 && distance <= 64) g_msm_prefetch = (uint32_t)distance;
}
extern "C" int h2b_msm_get_prefetch(void) { return (int)g_msm_prefetch; }

extern "C" int h2b_msm_get_pair_rounds(void) { return g_msm_pair_rounds; }

// Batch-affine pairing rounds run before the XYZZ bucket accumulation
// (0..3; rounds above 0 are built with H2B_EXPERIMENTS=1 only, otherwise
// the setting stays 0).  Default 0: on B200 a pairing addition (forward pass, shared
// inversion, backward pass) measured about 0.5 ns per addition against
// 0.3 ns for an XYZZ mixed addition (2^20 points, witness scalar mix).
// Results are identical; speed and the workspace size differ (the
// workspace-size queries follow this setting).
extern "C" void h2b_msm_set_pair_rounds(int rounds) { msm_set_pair_rounds(rounds); }

// Number of nonzero signed window digits (= sorted entries = bucket
// additions) the MSM of these scalars performs; written to *d_count (u64).
// Used by the benchmark for its algorithmic work count, untimed.
namespace h2b {
__global__ void k_msm_count(const Fr* __restrict__ sc, uint64_t n, int c, int W, uint32_t H,
                            unsigned long long* __restrict__ cnt)
{
    unsigned long long local = 0;
    const uint32_t full = 1u << c;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint4 half[2];
        glv::decompose(from_mont(ldg(&sc[i])), half[0], half[1]);
        for (int h = 0; h < 2; h++) {
            uint32_t carry = 0;
            for (int w = 0; w < W; w++) {
                uint32_t v = window_bits(half[h], w * c, c) + carry;
                int32_t d = (v > H) ? (int32_t)v - (int32_t)full : (int32_t)v;
                carry = (v > H) ? 1u : 0u;
                if (d != 0) local++;
            }
        }
    }
    atomicAdd(cnt, local);
}
} // namespace h2b

extern "C" RustError h2b_msm_count_entries(const void* d_scalars, uint64_t n, void* d_count, cudaStream_t stream)
{
    MsmPlan p = msm_plan(n);
    H2B_CUDA(cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), stream));
    if (n == 0) return ok();
    k_msm_count<<<grid_for(n, 256, 148u * 8u), 256, 0, stream>>>((const Fr*)d_scalars, n, p.c, p.W, p.H,
                                                                (unsigned long long*)d_count);
    H2B_LAUNCHED("k_msm_count");
    return ok();
}

extern "C" int h2b_msm_window_bits(uint64_t n) { return msm_plan(n).c; }
