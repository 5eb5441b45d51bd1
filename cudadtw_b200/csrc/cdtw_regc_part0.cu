// All-windows register-band cDTW over consecutive windows, four windows per thread, W = 0..16
// (see cdtw_reg.cuh); one translation unit per band range for a parallel
// build.
#include "cdtw_reg.cuh"

namespace cdtw {

void regc_fill_part0(void** eu, void** mh) {
    RegCRange<0, kMaxReg4W, 4>::fill((RegCKernel*)eu, (RegCKernel*)mh);
}

}  // namespace cdtw
