// Banded DTW for wide bands with the band spread over a group of lanes
// ("lane-block" kernels).  Device code shared by the all-windows and the
// search launchers (cdtw_lane.cu).
//
// Reference: sparse_block_cdtw / dense_block_cdtw (include/cdtw.cuh:164-363)
// spread one window over W+2 threads and step anti-diagonals through shared
// memory with a __syncthreads per step.  Here a group of G lanes (a power of
// two) runs two windows together, row by row like the register-band kernel:
//
//   * The band of a row (band coordinate k = i - j + W in [0, 2W]) is cut into
//     G blocks of B cells; lane g keeps cells k in [gB, gB + B) of both
//     windows in registers.  The row recurrence
//       D[j][k] = cost(z_j, q_{j-W+k}) + min(D[j-1][k], D[j-1][k+1], D[j][k-1])
//     chains left to right inside a block; the two windows' chains interleave.
//   * The lanes run as a pipeline one row apart: at step t lane g works on
//     row r = t - g.  Its first cell's left input is lane g-1's last cell of
//     the same row, finished one step earlier (a shuffle at the end of each
//     step); its last cell's upper input is lane g+1's first cell of the row
//     above, finished earlier in the same step (a shuffle after cell 0).
//     Lane 0's left and lane G-1's upper inputs are +inf (band edges).
//   * Query values of a lane's block are read from four shifted copies of
//     the +inf-padded query in shared memory with 16-byte loads (each lane
//     picks the copy that aligns its own start); they serve both windows.
//   * G*B >= 2W+1: the cells k > 2W of lane G-1 are outside the band.  Only
//     k = 2W+1 is ever read by a band cell (as the upper input of k = 2W one
//     row later), so after each row it is set to +inf (a warp-uniform switch
//     on its slot); the others only feed each other.
//   * Rows before 0 (the pipeline's start) keep the virtual row -1
//     (D[-1][-1] = 0, +inf elsewhere) by selects; rows after M-1 (its end) are
//     computed on clamped samples and never read.  D[M-1][W] sits at slot
//     W mod B of lane W / B after step M-1 + W/B.
//   * Search: every 16 steps the group takes the minimum of its current cells
//     -- the cells of rows t-G+1 .. t form a staircase that every warping path
//     crosses -- plus the forward LB_Keogh terms of the rows after t (the
//     cumulative bound of UCR_DTW_BIN.cpp:336, :666-677), and a window whose
//     bound reaches the best-so-far stops counting.
#pragma once

#include "common.cuh"

#include <type_traits>

namespace cdtw {

// Arguments of the lane-block kernels.
struct LaneArgs {
    const float* x;
    const double* mu;
    const float* sigma;
    const float4* qpad4;  // QueryPack::qpad: 4 shifted copies, lq4 float4 each
    int lq4;
    int qoff[4];          // float4 offset of each copy in the block's shared memory
    const float2* qenv;   // query envelope (search)
    int M, W, G, lgG, Nw;
    int gW, cW;           // lane and slot of band cell k = W
    int cph;              // slot in lane G-1 of band cell k = 2W+1
    // all (or listed) windows
    const int32_t* idx;
    int L;
    float* out;
    // search over a candidate list
    const Cand* cands;
    const int* count;
    int* work;
    unsigned long long* key;
    HitSink sink;
};

constexpr int kLaneThreads = 256;
constexpr int kLaneBMin = 18;   // cells per lane and window: instantiated range
constexpr int kLaneBMax = 48;
constexpr int kLaneCheck = 16;  // steps between early-abandon checks (search)

namespace {

// Sets p[c] to max(p[c], lim) for a warp-uniform runtime slot c.
template <int B>
__device__ __forceinline__ void lane_raise_slot(float (&p0)[B + 1], float (&p1)[B + 1], int c,
                                                float lim) {
    switch (c) {
#define CDTW_LANE_CASE(n)                              \
    case n:                                            \
        if constexpr (n < B) {                         \
            p0[n] = fmaxf(p0[n], lim);                 \
            p1[n] = fmaxf(p1[n], lim);                 \
        }                                              \
        break;
        CDTW_LANE_CASE(0) CDTW_LANE_CASE(1) CDTW_LANE_CASE(2) CDTW_LANE_CASE(3)
        CDTW_LANE_CASE(4) CDTW_LANE_CASE(5) CDTW_LANE_CASE(6) CDTW_LANE_CASE(7)
        CDTW_LANE_CASE(8) CDTW_LANE_CASE(9) CDTW_LANE_CASE(10) CDTW_LANE_CASE(11)
        CDTW_LANE_CASE(12) CDTW_LANE_CASE(13) CDTW_LANE_CASE(14) CDTW_LANE_CASE(15)
        CDTW_LANE_CASE(16) CDTW_LANE_CASE(17) CDTW_LANE_CASE(18) CDTW_LANE_CASE(19)
        CDTW_LANE_CASE(20) CDTW_LANE_CASE(21) CDTW_LANE_CASE(22) CDTW_LANE_CASE(23)
        CDTW_LANE_CASE(24) CDTW_LANE_CASE(25) CDTW_LANE_CASE(26) CDTW_LANE_CASE(27)
        CDTW_LANE_CASE(28) CDTW_LANE_CASE(29) CDTW_LANE_CASE(30) CDTW_LANE_CASE(31)
        CDTW_LANE_CASE(32) CDTW_LANE_CASE(33) CDTW_LANE_CASE(34) CDTW_LANE_CASE(35)
        CDTW_LANE_CASE(36) CDTW_LANE_CASE(37) CDTW_LANE_CASE(38) CDTW_LANE_CASE(39)
        CDTW_LANE_CASE(40) CDTW_LANE_CASE(41) CDTW_LANE_CASE(42) CDTW_LANE_CASE(43)
        CDTW_LANE_CASE(44) CDTW_LANE_CASE(45) CDTW_LANE_CASE(46) CDTW_LANE_CASE(47)
        CDTW_LANE_CASE(48) CDTW_LANE_CASE(49) CDTW_LANE_CASE(50) CDTW_LANE_CASE(51)
#undef CDTW_LANE_CASE
        default:
            break;
    }
}

// Reads p0[c], p1[c] for a warp-uniform runtime slot c.
template <int B>
__device__ __forceinline__ void lane_read_slot(const float (&p0)[B + 1], const float (&p1)[B + 1],
                                               int c, float& r0, float& r1) {
    switch (c) {
#define CDTW_LANE_CASE(n)      \
    case n:                    \
        if constexpr (n < B) { \
            r0 = p0[n];        \
            r1 = p1[n];        \
        }                      \
        break;
        CDTW_LANE_CASE(0) CDTW_LANE_CASE(1) CDTW_LANE_CASE(2) CDTW_LANE_CASE(3)
        CDTW_LANE_CASE(4) CDTW_LANE_CASE(5) CDTW_LANE_CASE(6) CDTW_LANE_CASE(7)
        CDTW_LANE_CASE(8) CDTW_LANE_CASE(9) CDTW_LANE_CASE(10) CDTW_LANE_CASE(11)
        CDTW_LANE_CASE(12) CDTW_LANE_CASE(13) CDTW_LANE_CASE(14) CDTW_LANE_CASE(15)
        CDTW_LANE_CASE(16) CDTW_LANE_CASE(17) CDTW_LANE_CASE(18) CDTW_LANE_CASE(19)
        CDTW_LANE_CASE(20) CDTW_LANE_CASE(21) CDTW_LANE_CASE(22) CDTW_LANE_CASE(23)
        CDTW_LANE_CASE(24) CDTW_LANE_CASE(25) CDTW_LANE_CASE(26) CDTW_LANE_CASE(27)
        CDTW_LANE_CASE(28) CDTW_LANE_CASE(29) CDTW_LANE_CASE(30) CDTW_LANE_CASE(31)
        CDTW_LANE_CASE(32) CDTW_LANE_CASE(33) CDTW_LANE_CASE(34) CDTW_LANE_CASE(35)
        CDTW_LANE_CASE(36) CDTW_LANE_CASE(37) CDTW_LANE_CASE(38) CDTW_LANE_CASE(39)
        CDTW_LANE_CASE(40) CDTW_LANE_CASE(41) CDTW_LANE_CASE(42) CDTW_LANE_CASE(43)
        CDTW_LANE_CASE(44) CDTW_LANE_CASE(45) CDTW_LANE_CASE(46) CDTW_LANE_CASE(47)
        CDTW_LANE_CASE(48) CDTW_LANE_CASE(49) CDTW_LANE_CASE(50) CDTW_LANE_CASE(51)
#undef CDTW_LANE_CASE
        default:
            break;
    }
}

// One row of the lane's block for both windows.  KEEP: rows before 0 keep
// the previous values (pipeline start).  Returns the cells' new values in
// p0 / p1; lin0 / lin1 are the left inputs of cell 0 (lane g-1's last cell of
// this row), and the upper input of the last cell comes from lane g+1.
template <int B, bool EU, bool KEEP>
__device__ __forceinline__ void lane_row(float (&p0)[B + 1], float (&p1)[B + 1], float z0,
                                         float z1, const float4* __restrict__ qrow, float lin0,
                                         float lin1, bool keep, bool last_lane, int G) {
    constexpr int NQ4 = (B + 3) / 4;
    float u0 = CDTW_INF, u1 = CDTW_INF;  // upper inputs of the last cell (lane g+1's cell 0)
    float l0 = lin0, l1 = lin1;          // left inputs
#pragma unroll
    for (int r4 = 0; r4 < NQ4; ++r4) {
        const float4 qq = qrow[r4];
        const float qv[4] = {qq.x, qq.y, qq.z, qq.w};
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int c = 4 * r4 + u;
            if (c < B) {
                const float up0 = (c == B - 1) ? u0 : p0[c + 1];
                const float up1 = (c == B - 1) ? u1 : p1[c + 1];
                float v0 = cell<EU>(z0 - qv[u], min3f(p0[c], up0, l0));
                float v1 = cell<EU>(z1 - qv[u], min3f(p1[c], up1, l1));
                if (KEEP && !keep) {  // row before 0: the virtual row stays
                    v0 = p0[c];
                    v1 = p1[c];
                }
                if (c == 0) {  // cell 0 is lane g-1's upper input for its last cell
                    u0 = __shfl_down_sync(0xffffffffu, v0, 1, G);
                    u1 = __shfl_down_sync(0xffffffffu, v1, 1, G);
                    if (last_lane) {
                        u0 = CDTW_INF;
                        u1 = CDTW_INF;
                    }
                }
                p0[c] = v0;
                p1[c] = v1;
                l0 = v0;
                l1 = v1;
            }
        }
    }
}

// cDTW of two windows (rows xw0 / xw1, normalisation n0 / n1) by the group
// of G lanes; lane g of the group calls with its g.  All 32 lanes of the warp
// call together (full-mask shuffles).  sq4: the query copies in shared
// memory.  SEARCH: alive0 / alive1 in, out (abandoned windows become dead;
// the warp stops when every window of the warp is dead), lbk0 / lbk1 the
// windows' forward LB_Keogh totals.  Results in r0 / r1 (valid in lane gW).
template <int B, bool EU, bool SEARCH>
__device__ __forceinline__ void lane_pair_dtw(const LaneArgs& a, const float4* sq4, int g,
                                              const float* __restrict__ xw0,
                                              const float* __restrict__ xw1, const Norm& n0,
                                              const Norm& n1, float lbk0, float lbk1,
                                              bool& alive0, bool& alive1, float& r0, float& r1) {
    const int M = a.M, G = a.G;
    const bool last_lane = g == G - 1;
    float p0[B + 1], p1[B + 1];
#pragma unroll
    for (int c = 0; c <= B; ++c) {
        const bool org = g == a.gW && c == a.cW;  // D[-1][-1] = 0 under cell k = W
        p0[c] = org ? 0.f : CDTW_INF;
        p1[c] = org ? 0.f : CDTW_INF;
    }
    float lin0 = CDTW_INF, lin1 = CDTW_INF;  // left inputs of cell 0
    float pre0 = 0.f, pre1 = 0.f;            // forward LB_Keogh of rows 0..t (lane 0)
    const float klim = last_lane ? CDTW_INF : -CDTW_INF;
    const int t_end = M - 1 + a.gW;
    const int bstep = g * (B - 1);
    // search: the samples of the next step's row (and lane 0's envelope
    // value of row t+1) are loaded one step ahead, the best-so-far
    // kLaneCheck / 2 steps before its check: the last survivors of a search
    // run nearly alone on their SMs and otherwise wait on these loads at every
    // step (all windows: enough warps hide them, and the extra work cost 7 %)
    float cx0 = 0.f, cx1 = 0.f, bsf_pf = CDTW_INF;
    float2 ce = make_float2(0.f, 0.f);
    if constexpr (SEARCH) {
        cx0 = __ldg(xw0 + min(max(-g, 0), M - 1));
        cx1 = __ldg(xw1 + min(max(-g, 0), M - 1));
        ce = __ldg(a.qenv);
    }
    auto step = [&](int t, auto keep_tag) {
        constexpr bool KEEP = decltype(keep_tag)::value;
        const int r = t - g;
        float x0, x1;
        if constexpr (SEARCH) {
            x0 = cx0;
            x1 = cx1;
            const int rn = min(max(r + 1, 0), M - 1);
            cx0 = __ldg(xw0 + rn);
            cx1 = __ldg(xw1 + rn);
        } else {
            const int rc = min(max(r, 0), M - 1);
            x0 = __ldg(xw0 + rc);
            x1 = __ldg(xw1 + rc);
        }
        const float z0 = znorm(n0, x0);
        const float z1 = znorm(n1, x1);
        if constexpr (SEARCH) {  // lane 0's row t: its forward LB_Keogh term
            const float2 e = ce;
            ce = __ldg(a.qenv + min(t + 1, M - 1));
            if ((t & (kLaneCheck - 1)) == kLaneCheck / 2 - 1) bsf_pf = load_bsf(a.key);
            if (t < M) {
                const float d0 = max3f(z0 - e.y, e.x - z0, 0.f);
                const float d1 = max3f(z1 - e.y, e.x - z1, 0.f);
                pre0 += EU ? d0 * d0 : d0;
                pre1 += EU ? d1 * d1 : d1;
            }
        }
        const int b = t + bstep;
        const float4* qrow = sq4 + a.qoff[b & 3] + (b >> 2);
        lane_row<B, EU, KEEP>(p0, p1, z0, z1, qrow, lin0, lin1, r >= 0, last_lane, G);
        lane_raise_slot<B>(p0, p1, a.cph, klim);  // k = 2W+1 stays outside the band
        lin0 = __shfl_up_sync(0xffffffffu, p0[B - 1], 1, G);
        lin1 = __shfl_up_sync(0xffffffffu, p1[B - 1], 1, G);
        if (g == 0) {
            lin0 = CDTW_INF;
            lin1 = CDTW_INF;
        }
    };
    int t = 0;
    for (; t < G - 1 && t <= t_end; ++t) step(t, std::true_type{});
    for (; t <= t_end; ++t) {
        step(t, std::false_type{});
        if constexpr (SEARCH) {
            if ((t & (kLaneCheck - 1)) == kLaneCheck - 1 && t < M - 1) {
                // staircase minimum of the group + LB_Keogh of rows t+1..M-1
                float m0 = p0[0], m1 = p1[0];
#pragma unroll
                for (int c = 1; c + 1 < B; c += 2) {
                    m0 = min3f(m0, p0[c], p0[c + 1]);
                    m1 = min3f(m1, p1[c], p1[c + 1]);
                }
                if ((B & 1) == 0) {
                    m0 = fminf(m0, p0[B - 1]);
                    m1 = fminf(m1, p1[B - 1]);
                }
                for (int o = 1; o < G; o <<= 1) {
                    m0 = fminf(m0, __shfl_xor_sync(0xffffffffu, m0, o, G));
                    m1 = fminf(m1, __shfl_xor_sync(0xffffffffu, m1, o, G));
                }
                const float q0 = __shfl_sync(0xffffffffu, pre0, 0, G);
                const float q1 = __shfl_sync(0xffffffffu, pre1, 0, G);
                const float bsf = bsf_pf;  // read kLaneCheck / 2 steps ago: at most larger
                alive0 = alive0 && (m0 + lb_suffix(lbk0, q0, M) * kLbSlack < bsf);
                alive1 = alive1 && (m1 + lb_suffix(lbk1, q1, M) * kLbSlack < bsf);
                if (!__any_sync(0xffffffffu, alive0 || alive1)) {
                    r0 = CDTW_INF;
                    r1 = CDTW_INF;
                    return;
                }
            }
        }
    }
    r0 = CDTW_INF;
    r1 = CDTW_INF;
    lane_read_slot<B>(p0, p1, a.cW, r0, r1);
}

// Loads the query copies into shared memory, copy c at a.qoff[c].
__device__ __forceinline__ void lane_stage_query(const LaneArgs& a, float4* sq4) {
    for (int e = threadIdx.x; e < 4 * a.lq4; e += blockDim.x) {
        const int c = e / a.lq4;
        sq4[a.qoff[c] + (e - c * a.lq4)] = a.qpad4[e];
    }
    __syncthreads();
}

// All (or listed) windows: group h of a warp runs listed windows 2u, 2u+1 of
// its unit u; a missing second window repeats the first and is not stored.
template <int B, bool EU>
__global__ void __launch_bounds__(kLaneThreads)
cdtw_lane_kernel(const LaneArgs a) {
    extern __shared__ float4 lsq4[];
    lane_stage_query(a, lsq4);
    const int G = a.G;
    const int g = threadIdx.x & (G - 1);
    const int64_t unit = ((int64_t)blockIdx.x * kLaneThreads + threadIdx.x) >> a.lgG;
    const int64_t units = div_up(a.L, 2);
    // a warp whose units all lie past the list has nothing to do
    const int64_t unit0 = ((int64_t)blockIdx.x * kLaneThreads + (threadIdx.x & ~31)) >> a.lgG;
    if (unit0 >= units) return;
    const bool live = unit < units;
    const int64_t t0 = live ? 2 * unit : 0;
    const int64_t t1 = live ? min(2 * unit + 1, (int64_t)a.L - 1) : 0;
    int w0 = a.idx ? a.idx[t0] : (int)t0;
    int w1 = a.idx ? a.idx[t1] : (int)t1;
    const bool ok0 = w0 >= 0 && w0 < a.Nw, ok1 = w1 >= 0 && w1 < a.Nw;
    if (!ok0) w0 = 0;  // a listed window outside the subject: NaN, no access
    if (!ok1) w1 = 0;
    const Norm n0 = make_norm(a.mu[w0], a.sigma[w0]);
    const Norm n1 = make_norm(a.mu[w1], a.sigma[w1]);
    bool al0 = true, al1 = true;
    float r0, r1;
    lane_pair_dtw<B, EU, false>(a, lsq4, g, a.x + w0, a.x + w1, n0, n1, 0.f, 0.f, al0, al1, r0,
                                r1);
    if (live && g == a.gW) {
        a.out[t0] = ok0 ? r0 : __int_as_float(0x7fc00000);
        if (2 * unit + 1 < a.L) a.out[t1] = ok1 ? r1 : __int_as_float(0x7fc00000);
    }
}

// Search over a candidate list: persistent warps take 64/G candidates at a
// time (two per group), skip those whose bound already exceeds the
// best-so-far, run the lane-block cDTW with early abandoning, and fold the
// results into the packed (distance, window) key.
template <int B, bool EU>
__global__ void __launch_bounds__(kLaneThreads)
cdtw_lane_search_kernel(const LaneArgs a) {
    extern __shared__ float4 lsq4[];
    lane_stage_query(a, lsq4);
    const int G = a.G;
    const int lane = threadIdx.x & 31;
    const int g = lane & (G - 1);
    const int h = lane >> a.lgG;  // group in warp
    const int per_warp = 64 >> a.lgG;
    const int n = *(const volatile int*)a.count;
    for (;;) {
        int base = 0;
        if (lane == 0) base = atomicAdd(a.work, per_warp);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= n) break;
        const int i0 = base + 2 * h, i1 = base + 2 * h + 1;
        Cand c0, c1;
        c0.w = 0;
        c0.lb = CDTW_INF;
        c0.lbk = 0.f;
        c1 = c0;
        if (i0 < n) c0 = a.cands[i0];
        if (i1 < n) c1 = a.cands[i1];
        const float bsf = load_bsf(a.key);
        bool al0 = i0 < n && c0.lb * kLbSlack < bsf;
        bool al1 = i1 < n && c1.lb * kLbSlack < bsf;
        if (!__any_sync(0xffffffffu, al0 || al1)) continue;
        const Norm n0 = make_norm(a.mu[c0.w], a.sigma[c0.w]);
        const Norm n1 = make_norm(a.mu[c1.w], a.sigma[c1.w]);
        float r0, r1;
        lane_pair_dtw<B, EU, true>(a, lsq4, g, a.x + c0.w, a.x + c1.w, n0, n1, c0.lbk, c1.lbk,
                                   al0, al1, r0, r1);
        if (g == a.gW) {
            if (i0 < n && r0 < CDTW_INF) report_window(a.key, a.sink, r0, (uint32_t)c0.w);
            if (i1 < n && r1 < CDTW_INF) report_window(a.key, a.sink, r1, (uint32_t)c1.w);
        }
    }
}

}  // namespace

using LaneKernel = void (*)(const LaneArgs);

// Kernel tables for B = kLaneBMin..kLaneBMax, filled by cdtw_lane_part*.cu.
void lane_fill_part0(LaneKernel* eu, LaneKernel* mh, LaneKernel* seu, LaneKernel* smh);
void lane_fill_part1(LaneKernel* eu, LaneKernel* mh, LaneKernel* seu, LaneKernel* smh);
void lane_fill_part2(LaneKernel* eu, LaneKernel* mh, LaneKernel* seu, LaneKernel* smh);
void lane_fill_part3(LaneKernel* eu, LaneKernel* mh, LaneKernel* seu, LaneKernel* smh);

template <int LO, int HI>
struct LaneRange {
    static void fill(LaneKernel* eu, LaneKernel* mh, LaneKernel* seu, LaneKernel* smh) {
        if constexpr (LO <= HI) {
            eu[LO] = cdtw_lane_kernel<LO, true>;
            mh[LO] = cdtw_lane_kernel<LO, false>;
            seu[LO] = cdtw_lane_search_kernel<LO, true>;
            smh[LO] = cdtw_lane_search_kernel<LO, false>;
            LaneRange<LO + 1, HI>::fill(eu, mh, seu, smh);
        }
    }
};

}  // namespace cdtw
