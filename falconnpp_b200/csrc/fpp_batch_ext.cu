// fpp_batch_ext.cu — instances of the fused batched kernel that start from
// per-table probe lists computed by the exact FP32 hash kernel (kHashExt):
// probe cut, gather / dedupe, rerank and top-k only.  The fhtDim template
// argument only sizes shared-memory regions the hashing would use, so one
// value serves every index.
#include "fpp_batch_kernel.cuh"

namespace fpp {

template <int MODE, int VI, int VI32>
static KernelSel ext_pair(bool big) {
  return big ? kernel_ptr<256, MODE, VI, VI32, kHashExt, true>() : kernel_ptr<256, MODE, VI, VI32, kHashExt, false>();
}

KernelSel pick_kernel_ext(int mode, int d, bool big) {
  const int v32 = vi_of(d, 4);
  if (mode == kRowsF32) {
    if (v32 == 1) return ext_pair<kRowsF32, 1, 1>(big);
    if (v32 == 2) return ext_pair<kRowsF32, 2, 2>(big);
    return ext_pair<kRowsF32, 4, 4>(big);
  }
  if (mode == kRowsBF16) {
    if (v32 == 1) return ext_pair<kRowsBF16, 1, 1>(big);
    if (v32 == 2) return ext_pair<kRowsBF16, 1, 2>(big);
    return ext_pair<kRowsBF16, 1, 4>(big);
  }
  if (v32 == 1) return ext_pair<kRowsFP8, 1, 1>(big);
  if (v32 == 2) return ext_pair<kRowsFP8, 1, 2>(big);
  return ext_pair<kRowsFP8, 1, 4>(big);
}

}  // namespace fpp
