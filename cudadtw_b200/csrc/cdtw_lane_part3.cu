// Lane-block cDTW kernels for B = 42..48 cells per lane (one of four
// translation units of the instantiation range, compiled in parallel).
#include "cdtw_lane.cuh"

namespace cdtw {

void lane_fill_part3(LaneKernel* eu, LaneKernel* mh, LaneKernel* seu, LaneKernel* smh) {
    LaneRange<42, 48>::fill(eu, mh, seu, smh);
}

}  // namespace cdtw
