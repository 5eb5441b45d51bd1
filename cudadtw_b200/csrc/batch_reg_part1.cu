// Register-band batched main-pass kernels for bands W = 49..62 (see
// batch_reg.cuh); one translation unit per band range.
#include "batch_reg.cuh"

namespace cdtw {

void batch_reg_fill_part1(void** eu, void** mh) {
    BatchRegRange<49, 62>::fill((BatchRegKernel*)eu, (BatchRegKernel*)mh);
}

}  // namespace cdtw
