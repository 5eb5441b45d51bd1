// All-windows register-band cDTW over consecutive windows, two windows per thread, W = 32..48
// (see cdtw_reg.cuh); one translation unit per band range for a parallel
// build.
#include "cdtw_reg.cuh"

namespace cdtw {

void regc_fill_part2(void** eu, void** mh) {
    RegCRange<kMaxReg3W + 1, kMaxReg2W, 2>::fill((RegCKernel*)eu, (RegCKernel*)mh);
}

}  // namespace cdtw
