// Register-band cDTW kernels for bands W = 0..48 (see cdtw_reg.cuh); one
// translation unit per band range so the instantiations compile in parallel.
#include "cdtw_reg.cuh"

namespace cdtw {

void reg_fill_part0(void** eu, void** mh, void** seu, void** smh) {
    RegRange<0, 48>::fill((RegKernel*)eu, (RegKernel*)mh, (RegSearchKernel*)seu,
                           (RegSearchKernel*)smh);
}

}  // namespace cdtw
