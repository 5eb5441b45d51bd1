// Register-band batched main-pass kernels for bands W = 73..81 (see
// batch_reg.cuh); one translation unit per band range.
#include "batch_reg.cuh"

namespace cdtw {

void batch_reg_fill_part3(void** eu, void** mh) {
    BatchRegRange<73, 81>::fill((BatchRegKernel*)eu, (BatchRegKernel*)mh);
}

}  // namespace cdtw
