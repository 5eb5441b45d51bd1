// Register-band batched main-pass kernels for bands W = 82..89 (see
// batch_reg.cuh); one translation unit per band range.
#include "batch_reg.cuh"

namespace cdtw {

void batch_reg_fill_part4(void** eu, void** mh) {
    BatchRegRange<82, 89>::fill((BatchRegKernel*)eu, (BatchRegKernel*)mh);
}

}  // namespace cdtw
