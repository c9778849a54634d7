// fpp_batch_big.cu — big-list instances of the fused batched kernel: per-table
// probe lists, probes and gather prefixes in per-block global scratch, for
// qProbes > 1024, n_tables * probes per table > 1024 or more than 16 probes
// per layer (the reference's own operating points, e.g. L = 50 with qProbes
// 1000..10000, src/main.cpp:69-80, test/falconnpp.py:150-172).
#include "fpp_batch_kernel.cuh"

namespace fpp {

KernelSel pick_kernel_big(int fht, int mode, int d) {
  const int v32 = vi_of(d, 4);
  if (mode == kRowsF32) {
    if (v32 == 1) return pick_fht<kRowsF32, 1, 1, true>(fht);
    if (v32 == 2) return pick_fht<kRowsF32, 2, 2, true>(fht);
    return pick_fht<kRowsF32, 4, 4, true>(fht);
  }
  if (mode == kRowsBF16) {
    if (v32 == 1) return pick_fht<kRowsBF16, 1, 1, true>(fht);
    if (v32 == 2) return pick_fht<kRowsBF16, 1, 2, true>(fht);
    return pick_fht<kRowsBF16, 1, 4, true>(fht);
  }
  if (v32 == 1) return pick_fht<kRowsFP8, 1, 1, true>(fht);
  if (v32 == 2) return pick_fht<kRowsFP8, 1, 2, true>(fht);
  return pick_fht<kRowsFP8, 1, 4, true>(fht);
}

}  // namespace fpp
