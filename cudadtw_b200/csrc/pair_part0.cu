// Pairwise cDTW forward kernels for C = 1..4 band slots per lane (one of
// four translation units, compiled in parallel; see pair.cuh).
#include "pair.cuh"

namespace cdtw {

PairFwdK pair_fwd_part0(int C, bool eu, int dm) {
    switch (C) {
        case 1: return pick_fwd<1>(eu, dm);
        case 2: return pick_fwd<2>(eu, dm);
        case 3: return pick_fwd<3>(eu, dm);
        default: return pick_fwd<4>(eu, dm);
    }
}

}  // namespace cdtw
