// Register-band batched main-pass kernels for bands W = 90..96 (see
// batch_reg.cuh); one translation unit per band range.
#include "batch_reg.cuh"

namespace cdtw {

void batch_reg_fill_part5(void** eu, void** mh) {
    BatchRegRange<90, 96>::fill((BatchRegKernel*)eu, (BatchRegKernel*)mh);
}

}  // namespace cdtw
