// Four-window register-band cDTW kernels for bands W = 0..16 (see
// cdtw_reg.cuh).
#include "cdtw_reg.cuh"

namespace cdtw {

void reg4_fill_part0(void** eu, void** mh) {
    Reg4Range<0, kMaxReg4W>::fill((RegKernel*)eu, (RegKernel*)mh);
}

}  // namespace cdtw
