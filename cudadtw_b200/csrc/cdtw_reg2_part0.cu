// Two-window register-band cDTW kernels for bands W = 0..28 (see
// cdtw_reg.cuh); one translation unit per band range for a parallel build.
#include "cdtw_reg.cuh"

namespace cdtw {

void reg2_fill_part0(void** eu, void** mh) {
    Reg2Range<0, 28>::fill((RegKernel*)eu, (RegKernel*)mh);
}

}  // namespace cdtw
