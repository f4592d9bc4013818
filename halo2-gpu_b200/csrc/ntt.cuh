// Internal NTT interface (pass-size tuning knob used by the autotuner).
#pragma once

namespace h2b {
int ntt_pass_stages();
void ntt_set_pass_stages(int b);
} // namespace h2b
