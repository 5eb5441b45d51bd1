// Register-band main pass of the batched search: for one band W, persistent
// CTAs take (query, tile) items of the queries with that band, run the shared
// front stage (statistics, LB_Kim, LB_Keogh) and then the register-band cDTW
// (cdtw_reg.cuh) of the survivors, 32 per warp, with early abandoning.
// Instantiated per band in batch_reg_part*.cu.
#pragma once

#include "batch.cuh"
#include "cdtw_reg.cuh"

namespace cdtw {

namespace {

template <int W, bool EU>
__global__ void __launch_bounds__(kBatchThreads)
batch_reg_kernel(const BatchArgs b) {
    extern __shared__ __align__(16) unsigned char smem[];
    const TileSmem ts = carve_tile(smem, b.tmax, b.mmax);
    float4* sq4 = ts.tail;                             // 4 * lq4max
    float2* senv = (float2*)(sq4 + 4 * b.lq4max);      // mmax
    __shared__ int s_item, s_na, s_nb, s_next;
    const int tid = threadIdx.x, lane = tid & 31;
    int q, tile;
    while (next_item(b, &s_item, q, tile)) {
        if (tid == 0) s_na = s_nb = s_next = 0;
        const BatchQ& Q = b.qs[q];
        const int M = Q.sa.M;
        for (int e = tid; e < 4 * Q.lq4; e += kBatchThreads) sq4[e] = Q.qpad4[e];
        for (int e = tid; e < M; e += kBatchThreads) senv[e] = Q.env[e];
        const int t0 = tile * Q.T;
        const int Tq = min(Q.T, Q.Nw - t0);
        tile_front<EU>(b.x, Q, t0, Tq, ts, &s_na, &s_nb);
        const int nb = s_nb;
        for (;;) {
            int base = 0;
            if (lane == 0) base = atomicAdd(&s_next, 32);
            base = __shfl_sync(0xffffffffu, base, 0);
            if (base >= nb) break;
            const int i = base + lane;
            const int l = (i < nb) ? ts.lb_l[i] : ts.lb_l[0];
            bool alive = (i < nb) && (ts.lb_lb[i] * kLbSlack < load_bsf(Q.key));
            if (!__any_sync(0xffffffffu, alive)) continue;
            const Norm nm = make_norm(ts.mu[l], ts.sg[l]);
            const float lbk = (i < nb) ? ts.lb_k[i] : 0.f;
            const float res =
                reg_window_dtw<W, EU>(sq4, Q.lq4, senv, M, b.x + t0 + l, nm, lbk, alive, Q.key);
            if (i < nb && res < CDTW_INF) atomicMin(Q.key, pack_key(res, (uint32_t)(t0 + l)));
        }
    }
}

using BatchRegKernel = void (*)(const BatchArgs);

template <int LO, int HI>
struct BatchRegRange {
    static void fill(BatchRegKernel* eu, BatchRegKernel* mh) {
        if constexpr (LO <= HI) {
            eu[LO] = batch_reg_kernel<LO, true>;
            mh[LO] = batch_reg_kernel<LO, false>;
            BatchRegRange<LO + 1, HI>::fill(eu, mh);
        }
    }
};

}  // namespace

void batch_reg_fill_part0(void** eu, void** mh);
void batch_reg_fill_part1(void** eu, void** mh);
void batch_reg_fill_part2(void** eu, void** mh);
void batch_reg_fill_part3(void** eu, void** mh);
void batch_reg_fill_part4(void** eu, void** mh);
void batch_reg_fill_part5(void** eu, void** mh);

}  // namespace cdtw
