// Device structures and the shared front stage of the batched search
// (batch.cu: strip kernels and seed passes, batch_reg.cuh: register-band
// tile kernels, batch_host.cu: plan and graph).
#pragma once

#include "cdtw_strip.cuh"

namespace cdtw {

struct BatchQ {
    StripArgs sa;            // per-query strip fields + M, W, P (x set too)
    const float* zq;         // z-normalised query
    const float2* env;       // query envelope
    const float4* qpad4;     // padded shifted copies (register-band bucket only)
    int lq4;                 // float4 per qpad copy
    unsigned long long* key; // result key
    int R, T, Nw, ntiles;    // R: strip rows of the seed cDTW (and of the main pass
                             // for strip-bucket queries)
    int item0;               // first tile item of this query in the seed pass
    int chunk0;              // first seed chunk (32 seed groups) of this query
    int seed_group;          // tiles per seed group (the group's best LB_Kim is a seed)
    int lane_refill;         // strip cDTW: refill per lane (1) or per warp (0)
};

struct SeedRec {
    int w;
    float lb;
    double mu;
    float sg;
    int pad;
};

// One persistent launch: its queries (positions into qs through qsel), their
// tile items (prefix), and its item counter b.ctr[ctr_idx].
struct BatchArgs {
    const BatchQ* qs;
    const int* qsel;          // nq entries: query index of each position
    int nq;
    const int* item_prefix;   // nq+1: tile items per position, prefix
    const int* chunk_prefix;  // nq+1: seed chunks per position, prefix (seed cDTW)
    int n_items, n_chunks;
    int* ctr;
    int ctr_idx;
    SeedRec* seeds;           // one per seed-pass tile item (all queries)
    float* ring;              // per resident warp: ring_stride floats
    int ring_stride;
    const float* x;
    int tmax, mmax, lq4max;   // shared-memory sizing
};

size_t batch_smem_bytes(int tmax, int mmax, int lq4max);
int batch_grid(cdtw_handle h, bool euclid, size_t smem, int* blocks);
int batch_warps_per_block();
int launch_batch_seed(cdtw_handle h, const BatchArgs& a, const BatchArgs& c, bool euclid,
                      size_t smem, int blocks);
int launch_batch_strip(cdtw_handle h, const BatchArgs& b, bool euclid, size_t smem, int blocks);
// Register-band main pass for bucket W (batch_reg_part*.cu).
int launch_batch_reg(cdtw_handle h, const BatchArgs& b, int W, bool euclid, size_t smem,
                     int blocks);
int batch_reg_prepare(cdtw_handle h, int W, bool euclid, size_t smem, int* blocks);

namespace {

constexpr int kBatchWarps = 4;
constexpr int kBatchThreads = kBatchWarps * 32;

__device__ __forceinline__ int find_query(const int* prefix, int nq, int item) {
    int lo = 0, hi = nq;  // prefix[lo] <= item < prefix[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (prefix[mid] <= item) lo = mid;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_scan_d(double v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Mean / sigma of the Tq windows of the tile staged in xs (Tq + M - 1
// samples), FP64 sums with a per-warp shift slid 32 windows per round
// (the avg_std kernel's scheme, from shared memory).
__device__ void tile_stats(const float* xs, int Tq, int M, double* mu, float* sg) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int per = (Tq + kBatchWarps - 1) / kBatchWarps;
    const int a = wid * per, b = min(Tq, a + per);
    if (a >= b) return;
    const double c = (double)xs[a];
    double s1 = 0.0, s2 = 0.0;
    for (int k = lane; k < M; k += 32) {
        const double v = (double)xs[a + k] - c;
        s1 += v;
        s2 = fma(v, v, s2);
    }
    s1 = warp_sum_d(s1);
    s2 = warp_sum_d(s2);
    const double invM = 1.0 / (double)M;
    for (int r0 = a; r0 < b; r0 += 32) {
        const int l = r0 + lane;
        double d1 = 0.0, d2 = 0.0;
        if (l < b - 1) {
            const double vin = (double)xs[l + M] - c, vout = (double)xs[l] - c;
            d1 = vin - vout;
            d2 = vin * vin - vout * vout;
        }
        const double i1 = warp_scan_d(d1, lane), i2 = warp_scan_d(d2, lane);
        if (l < b) {
            const double w1 = s1 + (i1 - d1), w2 = s2 + (i2 - d2);
            const double m1 = w1 * invM, var = w2 * invM - m1 * m1;
            mu[l] = c + m1;
            sg[l] = var > 0.0 ? (float)sqrt(var) : 1.0f;
        }
        s1 += __shfl_sync(0xffffffffu, i1, 31);
        s2 += __shfl_sync(0xffffffffu, i2, 31);
    }
}

// Shared-memory work area of one tile item.
struct TileSmem {
    double* mu;   // tmax
    float* sg;    // tmax
    int* la;      // tmax: LB_Kim survivors (local window)
    float* la_lb; // tmax
    int* lb_l;    // tmax: LB_Keogh survivors (local window)
    float* lb_lb; // tmax: their best bound
    float* lb_k;  // tmax: their forward LB_Keogh
    float* xs;    // tmax + mmax: the tile's samples
    float4* tail; // what follows (16-byte aligned)
};

__device__ __forceinline__ TileSmem carve_tile(unsigned char* smem, int tmax, int mmax) {
    TileSmem t;
    t.mu = (double*)smem;
    t.sg = (float*)(t.mu + tmax);
    t.la = (int*)(t.sg + tmax);
    t.la_lb = (float*)(t.la + tmax);
    t.lb_l = (int*)(t.la_lb + tmax);
    t.lb_lb = (float*)(t.lb_l + tmax);
    t.lb_k = (float*)(t.lb_lb + tmax);
    t.xs = (float*)(t.lb_k + tmax);
    t.tail = (float4*)(((uintptr_t)(t.xs + tmax + mmax) + 15) & ~(uintptr_t)15);
    return t;
}

// Front stage of a main-pass tile item: stage the samples, window
// statistics, LB_Kim of every window against the best-so-far, LB_Keogh
// (query envelope, early exit per warp) of the survivors.  Leaves the final
// survivors in ts.lb_* and their count in *s_nb.  Whole CTA.
template <bool EU>
__device__ void tile_front(const float* __restrict__ x, const BatchQ& Q, int t0, int Tq,
                           const TileSmem& ts, int* s_na, int* s_nb) {
    const int tid = threadIdx.x, lane = tid & 31;
    const int M = Q.sa.M;
    for (int i = tid; i < Tq + M - 1; i += kBatchThreads) ts.xs[i] = __ldg(x + t0 + i);
    __syncthreads();
    tile_stats(ts.xs, Tq, M, ts.mu, ts.sg);
    __syncthreads();
    const float lim = load_bsf(Q.key) / kLbSlack;
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
        const bool keep = l < Tq && lb < lim;
        const unsigned mk = __ballot_sync(0xffffffffu, keep);
        if (mk) {
            int at = 0;
            if (lane == 0) at = atomicAdd(s_na, __popc(mk));
            at = __shfl_sync(0xffffffffu, at, 0);
            if (keep) {
                const int p = at + __popc(mk & ((1u << lane) - 1));
                ts.la[p] = l;
                ts.la_lb[p] = lb;
            }
        }
    }
    __syncthreads();
    const int na = *s_na;
    for (int base = (tid & ~31); base < na; base += kBatchThreads) {
        const int i = base + lane;
        const bool valid = i < na;
        const int l = valid ? ts.la[i] : 0;
        const Norm nm = make_norm(ts.mu[l], ts.sg[l]);
        float af = 0.f;
        for (int k0 = 0; k0 < M; k0 += 32) {
            const int k1 = min(k0 + 32, M);
            for (int k = k0; k < k1; ++k) {
                const float z = znorm(nm, ts.xs[l + k]);
                const float2 e = __ldg(Q.env + k);
                const float df = max3f(z - e.y, e.x - z, 0.f);
                af = EU ? fmaf(df, df, af) : af + df;
            }
            if (__all_sync(0xffffffffu, !valid || af >= lim)) break;
        }
        const float lb = valid ? fmaxf(ts.la_lb[i], af) : CDTW_INF;
        const bool keep = valid && lb < lim;
        const unsigned mk = __ballot_sync(0xffffffffu, keep);
        if (mk) {
            int at = 0;
            if (lane == 0) at = atomicAdd(s_nb, __popc(mk));
            at = __shfl_sync(0xffffffffu, at, 0);
            if (keep) {
                const int p = at + __popc(mk & ((1u << lane) - 1));
                ts.lb_l[p] = l;
                ts.lb_lb[p] = lb;
                ts.lb_k[p] = af;
            }
        }
    }
    __syncthreads();
}

// Next main-pass item of this launch for the CTA: returns false when done.
__device__ __forceinline__ bool next_item(const BatchArgs& b, int* s_item, int& q, int& tile) {
    __syncthreads();
    if (threadIdx.x == 0) *s_item = atomicAdd(b.ctr + b.ctr_idx, 1);
    __syncthreads();
    const int item = *s_item;
    if (item >= b.n_items) return false;
    const int pos = find_query(b.item_prefix, b.nq, item);
    q = b.qsel[pos];
    tile = item - b.item_prefix[pos];
    return true;
}

}  // namespace

}  // namespace cdtw
