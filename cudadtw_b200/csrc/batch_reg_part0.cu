// Register-band batched main-pass kernels for bands W = 0..48 (see
// batch_reg.cuh); one translation unit per band range.
#include "batch_reg.cuh"

namespace cdtw {

void batch_reg_fill_part0(void** eu, void** mh) {
    BatchRegRange<0, 48>::fill((BatchRegKernel*)eu, (BatchRegKernel*)mh);
}

}  // namespace cdtw
