// Optional per-kernel CUDA-event timing (off by default).  When enabled, a
// launcher brackets its dominant kernel with events on the launch stream;
// h2b_prof_read sums the elapsed times recorded since the last enable.
#pragma once
#include <cuda_runtime.h>

namespace h2b {

enum ProfId : int {
    PROF_MSM_ACCUMULATE = 0,
    PROF_MSM_TOTAL = 1,
    PROF_NTT_PASSES = 2,
    PROF_BATCH_INVERT = 3,
    PROF_QUOTIENT = 4,
    PROF_PERMUTE_SORT = 5,
    PROF_IDS = 8
};

bool prof_on();
void prof_begin(int id, cudaStream_t st);
void prof_end(int id, cudaStream_t st);

} // namespace h2b
