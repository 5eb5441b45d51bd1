// Two-window register-band cDTW kernels for bands W = 29..48 (see
// cdtw_reg.cuh); one translation unit per band range for a parallel build.
#include "cdtw_reg.cuh"

namespace cdtw {

void reg2_fill_part1(void** eu, void** mh) {
    Reg2Range<29, 48>::fill((RegKernel*)eu, (RegKernel*)mh);
}

}  // namespace cdtw
