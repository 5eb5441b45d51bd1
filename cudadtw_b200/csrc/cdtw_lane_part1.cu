// Lane-block cDTW kernels for B = 26..33 cells per lane (one of four
// translation units of the instantiation range, compiled in parallel).
#include "cdtw_lane.cuh"

namespace cdtw {

void lane_fill_part1(LaneKernel* eu, LaneKernel* mh, LaneKernel* seu, LaneKernel* smh) {
    LaneRange<26, 33>::fill(eu, mh, seu, smh);
}

}  // namespace cdtw
