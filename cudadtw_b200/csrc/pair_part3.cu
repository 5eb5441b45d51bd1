// Pairwise cDTW forward kernels for C = 13..16 band slots per lane (one of
// four translation units, compiled in parallel; see pair.cuh).
#include "pair.cuh"

namespace cdtw {

PairFwdK pair_fwd_part3(int C, bool eu, int dm) {
    switch (C) {
        case 13: return pick_fwd<13>(eu, dm);
        case 14: return pick_fwd<14>(eu, dm);
        case 15: return pick_fwd<15>(eu, dm);
        default: return pick_fwd<16>(eu, dm);
    }
}

}  // namespace cdtw
