// fpp_batch_bf16.cu — BF16-rerank instances of the fused batched kernel.
#include "fpp_batch_kernel.cuh"

namespace fpp {

KernelSel pick_kernel_bf16(int fht, int d) {
  const int v = vi_of(d, 8), v32 = vi_of(d, 4);
  if (v == 1 && v32 == 1) return pick_fht<kRowsBF16, 1, 1>(fht);
  if (v == 1 && v32 == 2) return pick_fht<kRowsBF16, 1, 2>(fht);
  if (v == 2 && v32 == 4) return pick_fht<kRowsBF16, 2, 4>(fht);
  return KernelSel{nullptr, 0};
}

}  // namespace fpp
