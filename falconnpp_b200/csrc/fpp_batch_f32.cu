// fpp_batch_f32.cu — FP32 instances of the fused batched kernel (bit-exact with the plain path).
#include "fpp_batch_kernel.cuh"

namespace fpp {

KernelSel pick_kernel_f32(int fht, int d) {
  switch (vi_of(d, 4)) {
    case 1: return pick_fht<kRowsF32, 1, 1>(fht);
    case 2: return pick_fht<kRowsF32, 2, 2>(fht);
    default: return pick_fht<kRowsF32, 4, 4>(fht);
  }
}

}  // namespace fpp
