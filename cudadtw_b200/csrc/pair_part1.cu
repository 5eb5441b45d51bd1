// Pairwise cDTW forward kernels for C = 5..8 band slots per lane (one of
// four translation units, compiled in parallel; see pair.cuh).
#include "pair.cuh"

namespace cdtw {

PairFwdK pair_fwd_part1(int C, bool eu, int dm) {
    switch (C) {
        case 5: return pick_fwd<5>(eu, dm);
        case 6: return pick_fwd<6>(eu, dm);
        case 7: return pick_fwd<7>(eu, dm);
        default: return pick_fwd<8>(eu, dm);
    }
}

}  // namespace cdtw
