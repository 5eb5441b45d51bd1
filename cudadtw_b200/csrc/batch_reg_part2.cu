// Register-band batched main-pass kernels for bands W = 63..72 (see
// batch_reg.cuh); one translation unit per band range.
#include "batch_reg.cuh"

namespace cdtw {

void batch_reg_fill_part2(void** eu, void** mh) {
    BatchRegRange<63, 72>::fill((BatchRegKernel*)eu, (BatchRegKernel*)mh);
}

}  // namespace cdtw
