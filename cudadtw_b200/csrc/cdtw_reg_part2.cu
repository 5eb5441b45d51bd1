// Register-band cDTW kernels for bands W = 63..72 (see cdtw_reg.cuh); one
// translation unit per band range so the instantiations compile in parallel.
#include "cdtw_reg.cuh"

namespace cdtw {

void reg_fill_part2(void** eu, void** mh, void** seu, void** smh) {
    RegRange<63, 72>::fill((RegKernel*)eu, (RegKernel*)mh, (RegSearchKernel*)seu,
                           (RegSearchKernel*)smh);
}

}  // namespace cdtw
