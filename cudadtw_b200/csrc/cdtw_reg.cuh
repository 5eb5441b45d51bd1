// Banded DTW with the whole band of one window in registers ("register band").
//
// Reference: sparse_block_cdtw / dense_block_cdtw (include/cdtw.cuh:164-363),
// which spread one window over W+2 threads and step the anti-diagonals through
// shared memory with a __syncthreads per step.  Windows are independent and
// there are millions of them, so here one thread owns one window and keeps
// the 2W+1 band cells of the current row in registers; the 32 lanes of a warp
// run 32 neighbouring windows in lockstep, so all lanes read the same query
// values (a shared-memory broadcast) and consecutive stream samples (one
// coalesced 128-byte load per row).
//
// Orientation: rows are window (data) positions j = 0..M-1, columns are query
// positions i, band coordinate k = i - j + W in [0, 2W].  The cell update
//   D[j][k] = cost(z_j, q_{j-W+k}) + min(D[j-1][k], D[j-1][k+1], D[j][k-1])
// is one FADD, one three-input FMNMX and one FFMA.  Query positions outside
// [0, M) are padded with +inf, which makes out-of-matrix cells +inf without
// any per-cell test.  The result D[M-1][W] equals the reference's
// penalty[...][M] (cdtw.cuh:83).
#pragma once

#include "common.cuh"

#include <algorithm>

namespace cdtw {

namespace {

constexpr int kRegBlock = 128;
constexpr int kMaxRegW = 96;

template <int W, bool EU>
__global__ void __launch_bounds__(kRegBlock)
cdtw_reg_kernel(const float* __restrict__ x, const double* __restrict__ mu,
                const float* __restrict__ sigma, const float4* __restrict__ qpad4, int lq4,
                int M, int Nw, const int32_t* __restrict__ idx, int L, float* __restrict__ out) {
    extern __shared__ float4 sq4[];
    for (int e = threadIdx.x; e < 4 * lq4; e += blockDim.x) sq4[e] = qpad4[e];
    __syncthreads();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= L) return;
    const int w = idx ? idx[t] : t;
    if (w < 0 || w >= Nw) {  // a listed window outside the subject: NaN, no access
        out[t] = __int_as_float(0x7fc00000);
        return;
    }
    const Norm nm = make_norm(mu[w], sigma[w]);
    const float* __restrict__ xw = x + w;

    constexpr int B = 2 * W + 1;
    constexpr int NQ4 = (B + 3) / 4;
    float prev[B + 1];
#pragma unroll
    for (int k = 0; k <= B; ++k) prev[k] = CDTW_INF;
    prev[W] = 0.0f;  // virtual D[-1][-1] = 0 (cdtw.cuh:35, :191)
    float res = CDTW_INF;

    for (int j0 = 0; j0 < M; j0 += 4) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int j = j0 + u;
            const float z = znorm(nm, __ldg(xw + min(j, M - 1)));
            const float4* qr = sq4 + u * lq4 + (j0 >> 2);
            float qv[NQ4 * 4];
#pragma unroll
            for (int r = 0; r < NQ4; ++r) {
                const float4 v = qr[r];
                qv[4 * r + 0] = v.x;
                qv[4 * r + 1] = v.y;
                qv[4 * r + 2] = v.z;
                qv[4 * r + 3] = v.w;
            }
            float left = CDTW_INF;
            float cur[B];
#pragma unroll
            for (int k = 0; k < B; ++k) {
                const float m = min3f(prev[k], prev[k + 1], left);
                left = cell<EU>(z - qv[k], m);
                cur[k] = left;
            }
            if (j == M - 1) res = cur[W];
#pragma unroll
            for (int k = 0; k < B; ++k) prev[k] = cur[k];
        }
    }
    out[t] = res;
}

// Two windows per thread: both read the same query band values at a row (the
// band of row j is q[j-W .. j+W] whatever the window), so the shared-memory
// query loads are paid once for 2(2W+1) cells, and the two windows' cell
// chains interleave (two independent min chains per thread).  Listed windows
// 2t and 2t+1; a missing second window computes a copy of the first and is
// not stored.
constexpr int kMaxReg2W = 48;

template <int W, bool EU>
__global__ void __launch_bounds__(kRegBlock, 1)
cdtw_reg2_kernel(const float* __restrict__ x, const double* __restrict__ mu,
                 const float* __restrict__ sigma, const float4* __restrict__ qpad4, int lq4,
                 int M, int Nw, const int32_t* __restrict__ idx, int L, float* __restrict__ out) {
    extern __shared__ float4 sq4[];
    for (int e = threadIdx.x; e < 4 * lq4; e += blockDim.x) sq4[e] = qpad4[e];
    __syncthreads();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (2 * t >= L) return;
    const int t1 = min(2 * t + 1, L - 1);
    int w0 = idx ? idx[2 * t] : 2 * t;
    int w1 = idx ? idx[t1] : t1;
    const bool ok0 = w0 >= 0 && w0 < Nw, ok1 = w1 >= 0 && w1 < Nw;
    if (!ok0) w0 = 0;  // a listed window outside the subject: NaN, no access
    if (!ok1) w1 = 0;
    const Norm n0 = make_norm(mu[w0], sigma[w0]);
    const Norm n1 = make_norm(mu[w1], sigma[w1]);
    const float* __restrict__ x0 = x + w0;
    const float* __restrict__ x1 = x + w1;

    constexpr int B = 2 * W + 1;
    constexpr int NQ4 = (B + 3) / 4;
    float p0[B + 1], p1[B + 1];
#pragma unroll
    for (int k = 0; k <= B; ++k) {
        p0[k] = CDTW_INF;
        p1[k] = CDTW_INF;
    }
    p0[W] = 0.0f;
    p1[W] = 0.0f;
    float r0 = CDTW_INF, r1 = CDTW_INF;

    for (int j0 = 0; j0 < M; j0 += 4) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int j = j0 + u;
            const int jc = min(j, M - 1);
            const float z0 = znorm(n0, __ldg(x0 + jc));
            const float z1 = znorm(n1, __ldg(x1 + jc));
            const float4* qr = sq4 + u * lq4 + (j0 >> 2);
            float qv[NQ4 * 4];
#pragma unroll
            for (int r = 0; r < NQ4; ++r) {
                const float4 v = qr[r];
                qv[4 * r + 0] = v.x;
                qv[4 * r + 1] = v.y;
                qv[4 * r + 2] = v.z;
                qv[4 * r + 3] = v.w;
            }
            float l0 = CDTW_INF, l1 = CDTW_INF;
#pragma unroll
            for (int k = 0; k < B; ++k) {
                const float m0 = min3f(p0[k], p0[k + 1], l0);
                const float m1 = min3f(p1[k], p1[k + 1], l1);
                l0 = cell<EU>(z0 - qv[k], m0);
                l1 = cell<EU>(z1 - qv[k], m1);
                p0[k] = l0;  // p[k] is not read again this row
                p1[k] = l1;
            }
            if (j == M - 1) {
                r0 = p0[W];
                r1 = p1[W];
            }
        }
    }
    out[2 * t] = ok0 ? r0 : __int_as_float(0x7fc00000);
    if (2 * t + 1 < L) out[2 * t + 1] = ok1 ? r1 : __int_as_float(0x7fc00000);
}

// Four windows per thread for narrow bands: the query band values of a row
// are loaded once for 4(2W+1) cells and four independent min chains
// interleave (listed windows 4t .. 4t+3; missing ones repeat the last listed
// window and are not stored).
constexpr int kMaxReg4W = 16;

template <int W, bool EU>
__global__ void __launch_bounds__(kRegBlock, 1)
cdtw_reg4_kernel(const float* __restrict__ x, const double* __restrict__ mu,
                 const float* __restrict__ sigma, const float4* __restrict__ qpad4, int lq4,
                 int M, int Nw, const int32_t* __restrict__ idx, int L, float* __restrict__ out) {
    extern __shared__ float4 sq4[];
    for (int e = threadIdx.x; e < 4 * lq4; e += blockDim.x) sq4[e] = qpad4[e];
    __syncthreads();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (4 * t >= L) return;
    constexpr int NW = 4;
    constexpr int B = 2 * W + 1;
    constexpr int NQ4 = (B + 3) / 4;
    Norm nm[NW];
    const float* xw[NW];
    bool ok[NW];
#pragma unroll
    for (int v = 0; v < NW; ++v) {
        const int tv = min(4 * t + v, L - 1);
        int w = idx ? idx[tv] : tv;
        ok[v] = w >= 0 && w < Nw;
        if (!ok[v]) w = 0;  // a listed window outside the subject: NaN, no access
        nm[v] = make_norm(mu[w], sigma[w]);
        xw[v] = x + w;
    }
    float p[NW][B + 1];
#pragma unroll
    for (int v = 0; v < NW; ++v) {
#pragma unroll
        for (int k = 0; k <= B; ++k) p[v][k] = CDTW_INF;
        p[v][W] = 0.0f;
    }
    float r[NW];
#pragma unroll
    for (int v = 0; v < NW; ++v) r[v] = CDTW_INF;
    for (int j0 = 0; j0 < M; j0 += 4) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int j = j0 + u;
            const int jc = min(j, M - 1);
            float z[NW];
#pragma unroll
            for (int v = 0; v < NW; ++v) z[v] = znorm(nm[v], __ldg(xw[v] + jc));
            const float4* qr = sq4 + u * lq4 + (j0 >> 2);
            float qv[NQ4 * 4];
#pragma unroll
            for (int q4 = 0; q4 < NQ4; ++q4) {
                const float4 a = qr[q4];
                qv[4 * q4 + 0] = a.x;
                qv[4 * q4 + 1] = a.y;
                qv[4 * q4 + 2] = a.z;
                qv[4 * q4 + 3] = a.w;
            }
            float l[NW];
#pragma unroll
            for (int v = 0; v < NW; ++v) l[v] = CDTW_INF;
#pragma unroll
            for (int k = 0; k < B; ++k) {
#pragma unroll
                for (int v = 0; v < NW; ++v) {
                    const float m = min3f(p[v][k], p[v][k + 1], l[v]);
                    l[v] = cell<EU>(z[v] - qv[k], m);
                    p[v][k] = l[v];  // p[v][k] is not read again this row
                }
            }
            if (j == M - 1) {
#pragma unroll
                for (int v = 0; v < NW; ++v) r[v] = p[v][W];
            }
        }
    }
#pragma unroll
    for (int v = 0; v < NW; ++v)
        if (4 * t + v < L) out[4 * t + v] = ok[v] ? r[v] : __int_as_float(0x7fc00000);
}

// All windows, NW consecutive ones per thread (windows NW t .. NW t + NW - 1,
// no index list): window v's sample at row j is x[NW t + v + j], so the NW
// windows of a thread read one sliding run of the stream.  Rows go in groups
// of four; a group needs NW + 3 consecutive samples, of which four are new:
// they are loaded one group ahead and the run is shifted by four at the end
// of the group.  Every group but the last runs without row-index clamps or
// result tests; the last (one to four rows) ends at row M - 1.
template <int W, bool EU, int NW>
__device__ __forceinline__ void regc_row(float (&p)[NW][2 * W + 2], const float (&z)[NW],
                                         const float4* qr) {
    constexpr int B = 2 * W + 1;
    constexpr int NQ4 = (B + 3) / 4;
    float qv[NQ4 * 4];
#pragma unroll
    for (int r = 0; r < NQ4; ++r) {
        const float4 a = qr[r];
        qv[4 * r + 0] = a.x;
        qv[4 * r + 1] = a.y;
        qv[4 * r + 2] = a.z;
        qv[4 * r + 3] = a.w;
    }
    float l[NW];
#pragma unroll
    for (int v = 0; v < NW; ++v) l[v] = CDTW_INF;
#pragma unroll
    for (int k = 0; k < B; ++k) {
#pragma unroll
        for (int v = 0; v < NW; ++v) {
            const float m = min3f(p[v][k], p[v][k + 1], l[v]);
            l[v] = cell<EU>(z[v] - qv[k], m);
            p[v][k] = l[v];  // p[v][k] is not read again this row
        }
    }
}

template <int W, bool EU, int NW>
__global__ void __launch_bounds__(kRegBlock, 1)
cdtw_regc_kernel(const float* __restrict__ x, const double* __restrict__ mu,
                 const float* __restrict__ sigma, const float4* __restrict__ qpad4, int lq4,
                 int M, int Nw, float* __restrict__ out) {
    extern __shared__ float4 sq4[];
    for (int e = threadIdx.x; e < 4 * lq4; e += blockDim.x) sq4[e] = qpad4[e];
    __syncthreads();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int w0 = t * NW;
    if (w0 >= Nw) return;
    constexpr int B = 2 * W + 1;
    constexpr int NX = NW + 3;  // samples of a group of four rows
    // the last thread's missing windows repeat window Nw - 1's statistics and
    // read clamped samples; they are not stored
    const int rem = Nw - 1 - w0;                 // windows after w0 (>= 0)
    const int xlast = rem + M - 1;               // last sample index from w0
    const float* __restrict__ xb = x + w0;
    Norm nm[NW];
#pragma unroll
    for (int v = 0; v < NW; ++v) {
        const int w = w0 + min(v, rem);
        nm[v] = make_norm(mu[w], sigma[w]);
    }
    float p[NW][B + 1];
#pragma unroll
    for (int v = 0; v < NW; ++v) {
#pragma unroll
        for (int k = 0; k <= B; ++k) p[v][k] = CDTW_INF;
        p[v][W] = 0.0f;
    }
    float xs[NX];
#pragma unroll
    for (int i = 0; i < NX; ++i) xs[i] = __ldg(xb + min(i, xlast));
    int j0 = 0;
    for (; j0 + 4 < M; j0 += 4) {
        float nx[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) nx[i] = __ldg(xb + min(j0 + NX + i, xlast));
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            float z[NW];
#pragma unroll
            for (int v = 0; v < NW; ++v) z[v] = znorm(nm[v], xs[u + v]);
            regc_row<W, EU, NW>(p, z, sq4 + u * lq4 + (j0 >> 2));
        }
#pragma unroll
        for (int i = 0; i + 4 < NX; ++i) xs[i] = xs[i + 4];
#pragma unroll
        for (int i = 0; i < 4; ++i) xs[NX - 4 + i] = nx[i];
    }
    float r[NW];
#pragma unroll
    for (int v = 0; v < NW; ++v) r[v] = CDTW_INF;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        if (j0 + u < M) {
            float z[NW];
#pragma unroll
            for (int v = 0; v < NW; ++v) z[v] = znorm(nm[v], xs[u + v]);
            regc_row<W, EU, NW>(p, z, sq4 + u * lq4 + (j0 >> 2));
            if (j0 + u == M - 1) {
#pragma unroll
                for (int v = 0; v < NW; ++v) r[v] = p[v][W];
            }
        }
    }
#pragma unroll
    for (int v = 0; v < NW; ++v)
        if (v <= rem) out[w0 + v] = r[v];
}

using RegCKernel = void (*)(const float*, const double*, const float*, const float4*, int, int,
                            int, float*);

// Windows per thread of the consecutive-window kernels (register budget: the
// three-window kernel spills from W = 32).
constexpr int kMaxReg3W = 31;
constexpr int regc_per_thread(int W) {
    return W <= kMaxReg4W ? 4 : (W <= kMaxReg3W ? 3 : 2);
}

template <int LO, int HI, int NW>
struct RegCRange {
    static void fill(RegCKernel* eu, RegCKernel* mh) {
        if constexpr (LO <= HI) {
            eu[LO] = cdtw_regc_kernel<LO, true, NW>;
            mh[LO] = cdtw_regc_kernel<LO, false, NW>;
            RegCRange<LO + 1, HI, NW>::fill(eu, mh);
        }
    }
};

// cDTW of one window (xw, normalisation nm) against the query whose padded
// copies sit in shared memory (sq4, lq4 float4 per copy) with its envelope
// senv, abandoning once the last row minimum plus the remaining suffix of the
// window's forward LB_Keogh lbk (the cumulative bound cb of
// UCR_DTW_BIN.cpp:666-677, :336) reaches the best-so-far in *key.  alive
// marks lanes still worth finishing; the warp stops when no lane is.  All 32
// lanes call together.  Returns +inf if the warp stopped early.
template <int W, bool EU>
__device__ __forceinline__ float reg_window_dtw(const float4* sq4, int lq4,
                                                const float2* senv, int M,
                                                const float* __restrict__ xw, const Norm& nm,
                                                float lbk, bool& alive,
                                                const unsigned long long* key) {
    constexpr int B = 2 * W + 1;
    constexpr int NQ4 = (B + 3) / 4;
    float prev[B + 1];
#pragma unroll
    for (int k = 0; k <= B; ++k) prev[k] = CDTW_INF;
    prev[W] = 0.0f;
    float res = CDTW_INF, pre = 0.f;
    // W <= 64: the samples of the next 4-row group are loaded one group ahead
    // (with few windows in flight their latency is not hidden by other warps;
    // wider bands leave no registers for it)
    constexpr bool kAhead = W <= 64;
    float xn[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) xn[u] = kAhead ? __ldg(xw + min(u, M - 1)) : 0.f;
    for (int j0 = 0; j0 < M; j0 += 4) {
        float xc[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if constexpr (kAhead) {
                xc[u] = xn[u];
                xn[u] = __ldg(xw + min(j0 + 4 + u, M - 1));
            } else {
                xc[u] = __ldg(xw + min(j0 + u, M - 1));
            }
        }
        const bool check = (j0 & 7) == 4 && j0 + 3 < M - 1;  // rows j0..j0+3 are all real rows
        // W <= 64: the best-so-far is read before the group's cells
        const float bsf_early = (kAhead && check) ? load_bsf(key) : 0.f;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int j = j0 + u;
            const int jc = min(j, M - 1);
            const float z = znorm(nm, xc[u]);
            // forward LB_Keogh term of this data row (query envelope at j)
            const float2 e = senv[jc];
            const float dl = max3f(z - e.y, e.x - z, 0.f);
            pre += (j < M) ? (EU ? dl * dl : dl) : 0.f;
            const float4* qr = sq4 + u * lq4 + (j0 >> 2);
            float qv[NQ4 * 4];
#pragma unroll
            for (int r = 0; r < NQ4; ++r) {
                const float4 v = qr[r];
                qv[4 * r + 0] = v.x;
                qv[4 * r + 1] = v.y;
                qv[4 * r + 2] = v.z;
                qv[4 * r + 3] = v.w;
            }
            float left = CDTW_INF;
            float cur[B];
#pragma unroll
            for (int k = 0; k < B; ++k) {
                const float m = min3f(prev[k], prev[k + 1], left);
                left = cell<EU>(z - qv[k], m);
                cur[k] = left;
            }
            if (j == M - 1) res = cur[W];
#pragma unroll
            for (int k = 0; k < B; ++k) prev[k] = cur[k];
        }
        if (check) {
            float rmin = prev[0];
#pragma unroll
            for (int k = 1; k < B; k += 2) rmin = min3f(rmin, prev[k], prev[k + 1]);
            alive = alive && (rmin + lb_suffix(lbk, pre, M) * kLbSlack <
                              (kAhead ? bsf_early : load_bsf(key)));
            if (!__any_sync(0xffffffffu, alive)) return CDTW_INF;
        }
    }
    return res;
}

// Search variant: persistent warps take 32 candidates at a time from a device
// list, skip those whose lower bound already exceeds the best-so-far, run the
// register-band DTW with early abandoning, and fold results into *key by a
// packed (distance, window) atomicMin, so ties keep the lowest window (or
// append them to a hit list, report_window).
template <int W, bool EU>
__global__ void __launch_bounds__(kRegBlock)
cdtw_reg_search_kernel(const float* __restrict__ x, const double* __restrict__ mu,
                       const float* __restrict__ sigma, const float4* __restrict__ qpad4, int lq4,
                       const float2* __restrict__ qenv, int M, const Cand* __restrict__ cands,
                       const int* __restrict__ count, int* __restrict__ work,
                       unsigned long long* __restrict__ key, const HitSink sink) {
    extern __shared__ float4 sq4[];
    float2* senv = (float2*)(sq4 + 4 * lq4);
    for (int e = threadIdx.x; e < 4 * lq4; e += blockDim.x) sq4[e] = qpad4[e];
    for (int e = threadIdx.x; e < M; e += blockDim.x) senv[e] = qenv[e];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int n = *(const volatile int*)count;
    for (;;) {
        int base = 0;
        if (lane == 0) base = atomicAdd(work, 32);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= n) break;
        const int i = base + lane;
        Cand c;
        c.w = 0;
        c.lb = CDTW_INF;
        c.lbk = 0.f;
        if (i < n) c = cands[i];
        bool alive = (i < n) && (c.lb * kLbSlack < load_bsf(key));
        if (!__any_sync(0xffffffffu, alive)) continue;
        const Norm nm = make_norm(mu[c.w], sigma[c.w]);
        const float res = reg_window_dtw<W, EU>(sq4, lq4, senv, M, x + c.w, nm, c.lbk, alive, key);
        if (i < n && res < CDTW_INF) report_window(key, sink, res, (uint32_t)c.w);
    }
}

using RegKernel = void (*)(const float*, const double*, const float*, const float4*, int, int,
                           int, const int32_t*, int, float*);
using RegSearchKernel = void (*)(const float*, const double*, const float*, const float4*, int,
                                 const float2*, int, const Cand*, const int*, int*,
                                 unsigned long long*, const HitSink);

// Instantiates the kernels for bands LO..HI into the dispatch tables.
template <int LO, int HI>
struct RegRange {
    static void fill(RegKernel* eu, RegKernel* mh, RegSearchKernel* seu, RegSearchKernel* smh) {
        if constexpr (LO <= HI) {
            eu[LO] = cdtw_reg_kernel<LO, true>;
            mh[LO] = cdtw_reg_kernel<LO, false>;
            seu[LO] = cdtw_reg_search_kernel<LO, true>;
            smh[LO] = cdtw_reg_search_kernel<LO, false>;
            RegRange<LO + 1, HI>::fill(eu, mh, seu, smh);
        }
    }
};

}  // namespace

template <int LO, int HI>
struct Reg2Range {
    static void fill(RegKernel* eu, RegKernel* mh) {
        if constexpr (LO <= HI) {
            eu[LO] = cdtw_reg2_kernel<LO, true>;
            mh[LO] = cdtw_reg2_kernel<LO, false>;
            Reg2Range<LO + 1, HI>::fill(eu, mh);
        }
    }
};

template <int LO, int HI>
struct Reg4Range {
    static void fill(RegKernel* eu, RegKernel* mh) {
        if constexpr (LO <= HI) {
            eu[LO] = cdtw_reg4_kernel<LO, true>;
            mh[LO] = cdtw_reg4_kernel<LO, false>;
            Reg4Range<LO + 1, HI>::fill(eu, mh);
        }
    }
};

// Defined in cdtw_reg_part*.cu: each fills its range of bands.
void reg_fill_part0(void** eu, void** mh, void** seu, void** smh);
void reg_fill_part1(void** eu, void** mh, void** seu, void** smh);
void reg_fill_part2(void** eu, void** mh, void** seu, void** smh);
void reg_fill_part3(void** eu, void** mh, void** seu, void** smh);
void reg_fill_part4(void** eu, void** mh, void** seu, void** smh);
void reg_fill_part5(void** eu, void** mh, void** seu, void** smh);
void reg2_fill_part0(void** eu, void** mh);  // two-window kernels, cdtw_reg2_part*.cu
void reg2_fill_part1(void** eu, void** mh);
void reg4_fill_part0(void** eu, void** mh);  // four-window kernels, cdtw_reg4_part0.cu
// all-windows kernels over consecutive windows (cdtw_regc_part*.cu), windows
// per thread regc_per_thread(W)
void regc_fill_part0(void** eu, void** mh);
void regc_fill_part1(void** eu, void** mh);
void regc_fill_part2(void** eu, void** mh);

}  // namespace cdtw
