// All-windows register-band cDTW over consecutive windows, three windows per thread, W = 17..31
// (see cdtw_reg.cuh); one translation unit per band range for a parallel
// build.
#include "cdtw_reg.cuh"

namespace cdtw {

void regc_fill_part1(void** eu, void** mh) {
    RegCRange<kMaxReg4W + 1, kMaxReg3W, 3>::fill((RegCKernel*)eu, (RegCKernel*)mh);
}

}  // namespace cdtw
