// Batched subsequence search: hundreds of queries of uneven length and band
// against one stream, as (query, stream-tile) work items pulled from device
// queues by persistent CTAs.  No reference counterpart (the reference runs
// one query per process, GPU-dtw.cu).
//
// The host (batch_host.cu) captures into one CUDA graph:
//   A. seed pass    item = (query, tile of T windows): window statistics of
//                   the tile from its samples staged in shared memory (FP64
//                   sliding sums), LB_Kim of every window, and the tile's
//                   smallest bound as a seed window.
//   B. seed cDTW    the best seed of each group of tiles, for every query ->
//                   first best-so-far per query (packed (distance, window)
//                   key, atomicMin).
//   C. main pass    item = (query, tile): statistics, LB_Kim, LB_Keogh
//                   against the query envelope for the LB_Kim survivors
//                   (tile_front, batch.cuh), then the cDTW of the survivors
//                   by the CTA's warps with early abandoning against the live
//                   best-so-far.  One launch per bucket: the strip kernel here
//                   (any band), or the register-band kernel of one band W
//                   (batch_reg.cuh).
// The strip variant refills a warp either per group of 32 windows (lanes in
// lockstep) or per lane at strip boundaries (refill_dtw), chosen per query.
#include "batch.cuh"

#include <algorithm>

namespace cdtw {

namespace {

// cDTW of a list of windows by one warp.  get(idx, w, lb, lbk, nm) loads
// candidate idx; *next is the list cursor shared by the warps that work on
// the list.  LANE: a lane whose window finished or was abandoned takes the
// next candidate at the next strip boundary (lanes then sit at different
// strips and the query loads of a step diverge); otherwise the warp takes a
// new group of 32 only when all its lanes are done (lanes stay in lockstep
// and every query load is a broadcast).
template <int R, bool EU, bool LANE, class Get>
__device__ void refill_dtw(const BatchQ& Q, const float* __restrict__ x, int n, int* next,
                           Get get, float* ring) {
    const int lane = threadIdx.x & 31;
    const int M = Q.sa.M, P = Q.sa.P;
    const int S = (M + R - 1) / R;
    bool active = false;
    int w = 0, s = 0;
    float lbk = 0.f, pre = 0.f;
    Norm nm;
    nm.mhi = 0.f;
    nm.s = 1.f;
    nm.c = 0.f;
    for (;;) {
        const bool need = LANE ? !active : !__any_sync(0xffffffffu, active);
        const unsigned m = __ballot_sync(0xffffffffu, need);
        int base = 0;
        if (lane == 0 && m) base = atomicAdd(next, __popc(m));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (need) {
            const int idx = base + __popc(m & ((1u << lane) - 1));
            if (idx < n) {
                float lb;
                get(idx, w, lb, lbk, nm);
                if (lb * kLbSlack < load_bsf(Q.key)) {
                    s = 0;
                    pre = 0.f;
                    ring_reset(ring, P);
                    active = true;
                }
            }
        }
        if (!__any_sync(0xffffffffu, active)) {
            if (m != 0 && base >= n) break;  // list exhausted and nobody busy
            continue;
        }
        float rmin;
        const int j0 = active ? s * R : 0;
        strip_pass<R, EU, true>(Q.sa, x + w, nm, j0, ring, Q.env, pre, rmin);
        if (active) {
            if (s == S - 1) {
                atomicMin(Q.key, pack_key(strip_result<R>(Q.sa, ring), (uint32_t)w));
                active = false;
            } else if (rmin + lb_suffix(lbk, pre, M) * kLbSlack >= load_bsf(Q.key)) {
                active = false;  // abandoned
            } else {
                ++s;
            }
        }
    }
}

template <bool EU, class Get>
__device__ __forceinline__ void refill_dispatch(const BatchQ& Q, const float* x, int n, int* next,
                                                Get get, float* ring) {
    if (Q.lane_refill) {
        switch (Q.R) {
            case 16: refill_dtw<16, EU, true>(Q, x, n, next, get, ring); break;
            case 8: refill_dtw<8, EU, true>(Q, x, n, next, get, ring); break;
            case 4: refill_dtw<4, EU, true>(Q, x, n, next, get, ring); break;
            case 2: refill_dtw<2, EU, true>(Q, x, n, next, get, ring); break;
            default: refill_dtw<1, EU, true>(Q, x, n, next, get, ring); break;
        }
    } else {
        switch (Q.R) {
            case 16: refill_dtw<16, EU, false>(Q, x, n, next, get, ring); break;
            case 8: refill_dtw<8, EU, false>(Q, x, n, next, get, ring); break;
            case 4: refill_dtw<4, EU, false>(Q, x, n, next, get, ring); break;
            case 2: refill_dtw<2, EU, false>(Q, x, n, next, get, ring); break;
            default: refill_dtw<1, EU, false>(Q, x, n, next, get, ring); break;
        }
    }
}

__device__ __forceinline__ float* batch_ring(const BatchArgs& b) {
    const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    return b.ring + (size_t)gwarp * b.ring_stride + (threadIdx.x & 31);
}

// Pass A: statistics + LB_Kim per tile, the tile's smallest bound -> seed.
template <bool EU>
__global__ void __launch_bounds__(kBatchThreads)
batch_seed_kernel(const BatchArgs b) {
    extern __shared__ __align__(16) unsigned char smem[];
    const TileSmem ts = carve_tile(smem, b.tmax, b.mmax);
    __shared__ int s_item;
    __shared__ unsigned long long s_best;
    const int tid = threadIdx.x, lane = tid & 31;
    int q, tile;
    while (next_item(b, &s_item, q, tile)) {
        if (tid == 0) s_best = ~0ull;
        const BatchQ& Q = b.qs[q];
        const int t0 = tile * Q.T;
        const int Tq = min(Q.T, Q.Nw - t0);
        const int M = Q.sa.M;
        for (int i = tid; i < Tq + M - 1; i += kBatchThreads) ts.xs[i] = __ldg(b.x + t0 + i);
        __syncthreads();
        tile_stats(ts.xs, Tq, M, ts.mu, ts.sg);
        __syncthreads();
        for (int base = (tid & ~31); base < Tq; base += kBatchThreads) {
            const int l = base + lane;
            float lb = CDTW_INF;
            if (l < Tq) {
                const Norm nm = make_norm(ts.mu[l], ts.sg[l]);
                float sv[10], qv[10];
#pragma unroll
                for (int k = 0; k < 5; ++k) {
                    sv[k] = znorm(nm, ts.xs[l + k]);
                    qv[k] = __ldg(Q.zq + k);
                    sv[5 + k] = znorm(nm, ts.xs[l + M - 5 + k]);
                    qv[5 + k] = __ldg(Q.zq + M - 5 + k);
                }
                lb = lb_kim_dp<EU>(sv, qv);
            }
            // base is warp-uniform: every lane of the warp is here
            const unsigned long long k = warp_min_key(l < Tq && lb == lb, lb, (uint32_t)l);
            if (lane == 0 && k != ~0ull) atomicMin(&s_best, k);  // one per warp
        }
        __syncthreads();
        if (tid == 0) {
            SeedRec r;
            const int l = (s_best == ~0ull) ? 0 : (int)(uint32_t)s_best;
            r.w = t0 + l;
            r.lb = (s_best == ~0ull) ? CDTW_INF : key_dist(s_best);
            r.mu = ts.mu[l];
            r.sg = ts.sg[l];
            r.pad = 0;
            b.seeds[Q.item0 + tile] = r;
        }
    }
}

// Pass B: cDTW of each query's seeds (best of each seed group), one warp per
// chunk of 32 groups.
template <bool EU>
__global__ void __launch_bounds__(kBatchThreads)
batch_seed_dtw_kernel(const BatchArgs b) {
    __shared__ int s_next[kBatchWarps];
    float* ring = batch_ring(b);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (;;) {
        int chunk = 0;
        if (lane == 0) chunk = atomicAdd(b.ctr + b.ctr_idx, 1);
        chunk = __shfl_sync(0xffffffffu, chunk, 0);
        if (chunk >= b.n_chunks) break;
        const int pos = find_query(b.chunk_prefix, b.nq, chunk);
        const BatchQ& Q = b.qs[b.qsel[pos]];
        const int G = Q.seed_group;
        const int ngroups = (Q.ntiles + G - 1) / G;
        const int g0 = (chunk - b.chunk_prefix[pos]) * 32;
        const int n = min(32, ngroups - g0);
        if (lane == 0) s_next[wid] = 0;
        __syncwarp();
        auto get = [&](int idx, int& w, float& lb, float& lbk, Norm& nm) {
            // the group's tile seed with the smallest LB_Kim
            const int t0 = (g0 + idx) * G, t1 = min(Q.ntiles, t0 + G);
            SeedRec r = b.seeds[Q.item0 + t0];
            for (int t = t0 + 1; t < t1; ++t) {
                const SeedRec o = b.seeds[Q.item0 + t];
                if (o.lb < r.lb) r = o;
            }
            w = r.w;
            lb = (r.lb < CDTW_INF) ? 0.f : CDTW_INF;  // every real seed runs
            lbk = 0.f;                                 // no cumulative bound
            nm = make_norm(r.mu, r.sg);
        };
        refill_dispatch<EU>(Q, b.x, n, &s_next[wid], get, ring);
        __syncwarp();
    }
}

// Pass C, strip bucket: front stage, then the strip cDTW with lane refill.
template <bool EU>
__global__ void __launch_bounds__(kBatchThreads)
batch_strip_kernel(const BatchArgs b) {
    extern __shared__ __align__(16) unsigned char smem[];
    const TileSmem ts = carve_tile(smem, b.tmax, b.mmax);
    __shared__ int s_item, s_na, s_nb, s_next;
    float* ring = batch_ring(b);
    const int tid = threadIdx.x;
    int q, tile;
    while (next_item(b, &s_item, q, tile)) {
        if (tid == 0) s_na = s_nb = s_next = 0;
        const BatchQ& Q = b.qs[q];
        const int t0 = tile * Q.T;
        const int Tq = min(Q.T, Q.Nw - t0);
        tile_front<EU>(b.x, Q, t0, Tq, ts, &s_na, &s_nb);
        const int nb = s_nb;
        auto get = [&](int idx, int& w, float& lb, float& lbk, Norm& nm) {
            const int l = ts.lb_l[idx];
            w = t0 + l;
            lb = ts.lb_lb[idx];
            lbk = ts.lb_k[idx];
            nm = make_norm(ts.mu[l], ts.sg[l]);
        };
        if (nb > 0) refill_dispatch<EU>(Q, b.x, nb, &s_next, get, ring);
    }
}

}  // namespace

size_t batch_smem_bytes(int tmax, int mmax, int lq4max) {
    return (size_t)tmax * (8 + 4 * 6) + (size_t)(tmax + mmax) * 4 + 16 + (size_t)lq4max * 64 +
           (size_t)mmax * 8 + 64;
}

int batch_grid(cdtw_handle h, bool euclid, size_t smem, int* blocks) {
    const void* ks[3] = {
        euclid ? (const void*)batch_seed_kernel<true> : (const void*)batch_seed_kernel<false>,
        euclid ? (const void*)batch_strip_kernel<true> : (const void*)batch_strip_kernel<false>,
        euclid ? (const void*)batch_seed_dtw_kernel<true>
               : (const void*)batch_seed_dtw_kernel<false>};
    int best = 1 << 30;
    for (int i = 0; i < 3; ++i) {
        const size_t sm = (i == 2) ? 0 : smem;
        if (sm > 48 * 1024)
            CDTW_CUDA(h, cudaFuncSetAttribute(ks[i], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)sm));
        int per = 0;
        CDTW_CUDA(h, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, ks[i], kBatchThreads, sm));
        best = std::min(best, std::max(per, 1));
    }
    *blocks = best * h->sm_count;
    return CDTW_OK;
}

int batch_warps_per_block() { return kBatchWarps; }

int launch_batch_seed(cdtw_handle h, const BatchArgs& a, const BatchArgs& c, bool euclid,
                      size_t smem, int blocks) {
    if (euclid) batch_seed_kernel<true><<<blocks, kBatchThreads, smem, h->stream>>>(a);
    else batch_seed_kernel<false><<<blocks, kBatchThreads, smem, h->stream>>>(a);
    CDTW_LAUNCH(h, "batch_seed_kernel");
    if (euclid) batch_seed_dtw_kernel<true><<<blocks, kBatchThreads, 0, h->stream>>>(c);
    else batch_seed_dtw_kernel<false><<<blocks, kBatchThreads, 0, h->stream>>>(c);
    CDTW_LAUNCH(h, "batch_seed_dtw_kernel");
    return CDTW_OK;
}

int launch_batch_strip(cdtw_handle h, const BatchArgs& b, bool euclid, size_t smem, int blocks) {
    if (euclid) batch_strip_kernel<true><<<blocks, kBatchThreads, smem, h->stream>>>(b);
    else batch_strip_kernel<false><<<blocks, kBatchThreads, smem, h->stream>>>(b);
    CDTW_LAUNCH(h, "batch_strip_kernel");
    return CDTW_OK;
}

}  // namespace cdtw
