// Pairwise cDTW forward kernels for C = 9..12 band slots per lane (one of
// four translation units, compiled in parallel; see pair.cuh).
#include "pair.cuh"

namespace cdtw {

PairFwdK pair_fwd_part2(int C, bool eu, int dm) {
    switch (C) {
        case 9: return pick_fwd<9>(eu, dm);
        case 10: return pick_fwd<10>(eu, dm);
        case 11: return pick_fwd<11>(eu, dm);
        default: return pick_fwd<12>(eu, dm);
    }
}

}  // namespace cdtw
