// fpp_batch_fp8.cu — FP8-E4M3-rerank instances of the fused batched kernel.
#include "fpp_batch_kernel.cuh"

namespace fpp {

KernelSel pick_kernel_fp8(int fht, int d, bool tc_only) {
  // the first rerank runs on the tensor cores (VI unused); VI32 sizes the FP32 re-score
  const int v32 = vi_of(d, 4);
  if (tc_only && fht == 256) {
    if (v32 == 1) return kernel_ptr<256, kRowsFP8, 1, 1, kHashTC>();
    if (v32 == 2) return kernel_ptr<256, kRowsFP8, 1, 2, kHashTC>();
    return kernel_ptr<256, kRowsFP8, 1, 4, kHashTC>();
  }
  if (v32 == 1) return pick_fht<kRowsFP8, 1, 1>(fht);
  if (v32 == 2) return pick_fht<kRowsFP8, 1, 2>(fht);
  if (v32 == 4) return pick_fht<kRowsFP8, 1, 4>(fht);
  return KernelSel{nullptr, 0};
}

}  // namespace fpp
