// Register-band cDTW kernels for bands W = 82..89 (see cdtw_reg.cuh); one
// translation unit per band range so the instantiations compile in parallel.
#include "cdtw_reg.cuh"

namespace cdtw {

void reg_fill_part4(void** eu, void** mh, void** seu, void** smh) {
    RegRange<82, 89>::fill((RegKernel*)eu, (RegKernel*)mh, (RegSearchKernel*)seu,
                           (RegSearchKernel*)smh);
}

}  // namespace cdtw
