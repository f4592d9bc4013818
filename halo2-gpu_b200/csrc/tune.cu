// Per-size tuning table (no counterpart in the reference, whose MSM window
// width is a fixed formula of n, halo2_proofs/cuda/src/multiexp.cu:260-300,
// and whose NTT splits its stages by a fixed block_k,
// halo2_proofs/cuda/include/kernel/ntt_combine.h:90-94).
//
// The autotuner (halo2-gpu_b200/autotune.py) times candidate settings for
// each (parameter, log2 size) on the GPU it runs on and writes the winners
// here; the MSM planner (msm.cu, plain-base MSMs only: a window table's
// layout is fixed by the window width it was built with, and its long
// buckets want the chunk rule) and the NTT pass planner
// (ntt.cu) read them.  0 means "automatic" (the built-in formula).  Every
// setting gives the same results; only the time changes.  Workspace-size
// queries depend on the MSM entries, so set them before sizing scratch.
#include <atomic>
#include "abi.cuh"

namespace h2b {

constexpr int TUNE_PARAMS = 3;   // 0 MSM window bits, 1 MSM chunk entries, 2 NTT stages per pass
constexpr int TUNE_MAX_LOG = 32;
static std::atomic<int> g_tune[TUNE_PARAMS][TUNE_MAX_LOG + 1];

static bool tune_valid(uint32_t param, int32_t v)
{
    if (v == 0) return true;
    switch (param) {
    case 0: return v >= 10 && v <= 16;   // windows the default plans also use (sizes 2^10 .. 2^27)
    case 1: return v >= 8 && v <= 512;   // sorted entries per accumulation thread
    case 2: return v >= 1 && v <= 11;    // radix-2 stages per shared-memory pass (11: radix-4 passes only)
    default: return false;
    }
}

int tune_value(int param, int log_n)
{
    if (param < 0 || param >= TUNE_PARAMS || log_n < 0 || log_n > TUNE_MAX_LOG) return 0;
    return g_tune[param][log_n].load(std::memory_order_relaxed);
}

}  // namespace h2b

extern "C" int32_t h2b_tune_set(uint32_t param, uint32_t log_n, int32_t value)
{
    if (param >= (uint32_t)h2b::TUNE_PARAMS || log_n > (uint32_t)h2b::TUNE_MAX_LOG || !h2b::tune_valid(param, value))
        return -1;
    h2b::g_tune[param][log_n].store(value, std::memory_order_relaxed);
    return 0;
}

extern "C" int32_t h2b_tune_get(uint32_t param, uint32_t log_n)
{
    return h2b::tune_value((int)param, (int)log_n);
}

extern "C" void h2b_tune_clear(void)
{
    for (int p = 0; p < h2b::TUNE_PARAMS; p++)
        for (int l = 0; l <= h2b::TUNE_MAX_LOG; l++) h2b::g_tune[p][l].store(0, std::memory_order_relaxed);
}
