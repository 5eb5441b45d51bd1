// Windowed statistics of the stream and preparation of the query.
//
// Reference: include/stats.cuh.  The reference makes two FP64 prefix sums over
// the whole stream (CUB scans, 2 cudaMalloc + 5 kernels per 1e7-sample epoch,
// stats.cuh:85-142) and then takes the variance in FP32 (stats.cuh:49), which
// loses the variance of level-shifted signals.  Here one kernel reads the
// stream once: each warp owns a run of consecutive windows in four
// sub-runs, keeps FP64 sums of (x-c) and (x-c)^2 for a shift c per sub-run,
// and slides them 32 windows per round with warp scans of the
// entering-minus-leaving terms (the four sub-runs' scans interleaved).
// Output per window: mean (FP64) and sigma (FP32), 12 bytes.
#include "common.cuh"

namespace cdtw {

namespace {

constexpr int kStatsRounds = 64;                 // rounds of 32 windows per warp
constexpr int kStatsWarpWindows = 32 * kStatsRounds;
constexpr int kStatsBlock = 128;                 // 4 warps per block
constexpr int kStatsSub = 4;                     // interleaved sub-runs per warp

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <class XT, class ST>
__global__ void __launch_bounds__(kStatsBlock)
avg_std_kernel(const XT* __restrict__ x, int64_t N, int M, double* __restrict__ mu,
               ST* __restrict__ sigma) {
    // The warp's run of kStatsWarpWindows windows is split into kStatsSub
    // sub-runs, each with its own shift c and starting sums; their scans are
    // interleaved round by round (independent shuffle / FP64 chains).
    const int64_t Nw = N - M + 1;
    const int lane = threadIdx.x & 31;
    const int64_t warp = (int64_t)blockIdx.x * (kStatsBlock / 32) + (threadIdx.x >> 5);
    const int64_t a = warp * kStatsWarpWindows;
    if (a >= Nw) return;
    constexpr int kSubRounds = kStatsRounds / kStatsSub;
    constexpr int kSubWindows = 32 * kSubRounds;
    double c[kStatsSub], s1[kStatsSub], s2[kStatsSub];
#pragma unroll
    for (int u = 0; u < kStatsSub; ++u) {
        const int64_t as = min(a + (int64_t)u * kSubWindows, Nw - 1);
        c[u] = (double)x[as];
        s1[u] = 0.0;
        s2[u] = 0.0;
    }
    // sums of the first window of every sub-run
    for (int k = lane; k < M; k += 32) {
#pragma unroll
        for (int u = 0; u < kStatsSub; ++u) {
            const int64_t as = min(a + (int64_t)u * kSubWindows, Nw - 1);
            const double v = (double)x[as + k] - c[u];
            s1[u] += v;
            s2[u] = fma(v, v, s2[u]);
        }
    }
#pragma unroll
    for (int u = 0; u < kStatsSub; ++u) {
        s1[u] = warp_sum(s1[u]);
        s2[u] = warp_sum(s2[u]);
    }
    const double invM = 1.0 / (double)M;
    for (int r = 0; r < kSubRounds; ++r) {
        if (a + (int64_t)r * 32 >= Nw) break;  // warp-uniform (sub-run 0 ends first)
        double d1[kStatsSub], d2[kStatsSub];
        int64_t wv[kStatsSub];
#pragma unroll
        for (int u = 0; u < kStatsSub; ++u) {
            const int64_t w = a + (int64_t)u * kSubWindows + (int64_t)r * 32 + lane;
            wv[u] = w;
            d1[u] = 0.0;
            d2[u] = 0.0;
            if (w < Nw - 1) {
                // window w+1 = window w + x[w+M] - x[w]
                const double vin = (double)x[w + M] - c[u], vout = (double)x[w] - c[u];
                d1[u] = vin - vout;
                d2[u] = vin * vin - vout * vout;
            }
        }
        double i1[kStatsSub], i2[kStatsSub];
#pragma unroll
        for (int u = 0; u < kStatsSub; ++u) {
            i1[u] = d1[u];
            i2[u] = d2[u];
        }
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
            for (int u = 0; u < kStatsSub; ++u) {
                const double t1 = __shfl_up_sync(0xffffffffu, i1[u], o);
                const double t2 = __shfl_up_sync(0xffffffffu, i2[u], o);
                if (lane >= o) {
                    i1[u] += t1;
                    i2[u] += t2;
                }
            }
        }
#pragma unroll
        for (int u = 0; u < kStatsSub; ++u) {
            // sums of window w: base + exclusive scan
            const double w1 = s1[u] + (i1[u] - d1[u]), w2 = s2[u] + (i2[u] - d2[u]);
            if (wv[u] < Nw) {
                const double m1 = w1 * invM;
                const double var = w2 * invM - m1 * m1;
                mu[wv[u]] = c[u] + m1;
                sigma[wv[u]] = var > 0.0 ? (ST)sqrt(var) : (ST)1;
            }
            s1[u] += __shfl_sync(0xffffffffu, i1[u], 31);
            s2[u] += __shfl_sync(0xffffffffu, i2[u], 31);
        }
    }
}

// One block prepares the query pack: FP64 two-pass z-normalisation (the
// reference does this on the host in FP32, GPU-dtw.cu:67 / stats.cuh:8-28),
// the +inf-padded shifted copies read by the cDTW kernels, and the +-W
// envelope (same values as Lemire's filter, bounds.cuh:13-64).  Shared
// memory: M doubles (zs) and M floats behind them.
__device__ __forceinline__ void prepare_query_body(const float* __restrict__ qraw, int M, int W,
                                                   const QueryPack& p, double* zs) {
    float* zf = reinterpret_cast<float*>(zs + M);  // the z-values rounded to float
    __shared__ double red[2][8];
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
    double s = 0.0;
    for (int i = t; i < M; i += blockDim.x) {
        const double v = (double)qraw[i];
        zs[i] = v;
        s += v;
    }
    __syncthreads();  // qraw may be p.zq (a host query staged there)
    for (int i = t; p.qraw && i < M; i += blockDim.x) p.qraw[i] = (float)zs[i];
    s = warp_sum(s);
    if (lane == 0) red[0][wid] = s;
    __syncthreads();
    double tot = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) tot += red[0][k];
    const double mean = tot / M;
    double v2 = 0.0;
    for (int i = t; i < M; i += blockDim.x) {
        const double d = zs[i] - mean;
        v2 = fma(d, d, v2);
    }
    v2 = warp_sum(v2);
    if (lane == 0) red[1][wid] = v2;
    __syncthreads();
    double vt = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) vt += red[1][k];
    const double var = vt / M;
    const double sd = var > 0.0 ? sqrt(var) : 1.0;
    __syncthreads();
    for (int i = t; i < M; i += blockDim.x) {
        const double z = (zs[i] - mean) / sd;
        zs[i] = z;
        zf[i] = (float)z;
        p.zq64[i] = z;
        p.zq[i] = (float)z;
    }
    __syncthreads();
    // padded shifted copies: copy m, index a -> qp[a+m], qp[b] = zq[b-W]
    for (int e = t; p.qpad && e < 4 * p.lq; e += blockDim.x) {
        const int m = e / p.lq, a = e - m * p.lq;
        const int i = a + m - W;
        p.qpad[e] = (i >= 0 && i < M) ? (float)zs[i] : CDTW_INF;
    }
    // reversed extended copies for the strip kernel
    if (p.qrev) {
        const int lo = qrev_lo(W), A = p.qrev_base, len = qrev_hi(M, W) - lo + 1;
        for (int e = t; e < 4 * p.lqr; e += blockDim.x) {
            const int m = e / p.lqr, b = e - m * p.lqr + m;  // qr index
            float v = CDTW_INF;
            if (b < len) {
                const int i = A - b;
                v = (i < 0) ? CDTW_INF : (i < M ? (float)zs[i] : (float)i * 1e18f);
            }
            p.qrev[e] = v;
        }
    }
    // envelope over [k-W, k+W] clipped to the query, from the float values
    // (rounding is monotone: the extrema of the rounded values are the
    // rounded extrema); four independent min / max chains per window
    for (int k = t; k < M; k += blockDim.x) {
        const int a0 = max(0, k - W), a1 = min(M - 1, k + W);
        float lo[4], hi[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) lo[u] = hi[u] = zf[k];
        int i = a0;
        for (; i + 3 <= a1; i += 4) {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                lo[u] = fminf(lo[u], zf[i + u]);
                hi[u] = fmaxf(hi[u], zf[i + u]);
            }
        }
        for (; i <= a1; ++i) {
            lo[0] = fminf(lo[0], zf[i]);
            hi[0] = fmaxf(hi[0], zf[i]);
        }
        p.env[k] = make_float2(fminf(fminf(lo[0], lo[1]), fminf(lo[2], lo[3])),
                               fmaxf(fmaxf(hi[0], hi[1]), fmaxf(hi[2], hi[3])));
    }
}

__global__ void __launch_bounds__(256)
prepare_query_kernel(const float* __restrict__ qraw, int M, int W, QueryPack p) {
    extern __shared__ double zs[];  // M doubles, M floats
    prepare_query_body(qraw, M, W, p, zs);
}

__global__ void __launch_bounds__(256)
prepare_queries_kernel(const float* __restrict__ raw, const int64_t* __restrict__ offs,
                       const QueryPack* __restrict__ packs) {
    extern __shared__ double zs[];
    const QueryPack p = packs[blockIdx.x];
    prepare_query_body(raw + offs[blockIdx.x], p.M, p.W, p, zs);
}

}  // namespace

int launch_avg_std(cdtw_handle h, const float* x, int64_t N, int M, double* mu, float* sigma) {
    const int64_t Nw = N - M + 1;
    const int64_t warps = div_up(Nw, kStatsWarpWindows);
    const int64_t blocks = div_up(warps, kStatsBlock / 32);
    avg_std_kernel<float, float><<<(unsigned)blocks, kStatsBlock, 0, h->stream>>>(x, N, M, mu,
                                                                                  sigma);
    CDTW_LAUNCH(h, "avg_std_kernel");
    return CDTW_OK;
}

// FP64 sigma (ED and LDTW paths), float32 or float64 series.
int launch_avg_std64(cdtw_handle h, const float* x, int64_t N, int M, double* mu, double* sigma) {
    const int64_t blocks = div_up(div_up(N - M + 1, kStatsWarpWindows), kStatsBlock / 32);
    avg_std_kernel<float, double><<<(unsigned)blocks, kStatsBlock, 0, h->stream>>>(x, N, M, mu,
                                                                                   sigma);
    CDTW_LAUNCH(h, "avg_std_kernel");
    return CDTW_OK;
}
int launch_avg_std64(cdtw_handle h, const double* x, int64_t N, int M, double* mu, double* sigma) {
    const int64_t blocks = div_up(div_up(N - M + 1, kStatsWarpWindows), kStatsBlock / 32);
    avg_std_kernel<double, double><<<(unsigned)blocks, kStatsBlock, 0, h->stream>>>(x, N, M, mu,
                                                                                    sigma);
    CDTW_LAUNCH(h, "avg_std_kernel");
    return CDTW_OK;
}

int launch_prepare_queries(cdtw_handle h, const float* raw, const int64_t* offs,
                           const QueryPack* packs, int nq, int max_m) {
    const size_t smem = (size_t)max_m * (sizeof(double) + sizeof(float));
    if (smem > 48 * 1024)
        CDTW_CUDA(h, cudaFuncSetAttribute((const void*)prepare_queries_kernel,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
    prepare_queries_kernel<<<nq, 256, smem, h->stream>>>(raw, offs, packs);
    CDTW_LAUNCH(h, "prepare_queries_kernel");
    return CDTW_OK;
}

int launch_prepare_query(cdtw_handle h, const float* d_query_raw, int M, int W) {
    const size_t smem = (size_t)M * (sizeof(double) + sizeof(float));
    if (smem > 48 * 1024)
        CDTW_CUDA(h, cudaFuncSetAttribute((const void*)prepare_query_kernel,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
    prepare_query_kernel<<<1, 256, smem, h->stream>>>(d_query_raw, M, W, h->q);
    CDTW_LAUNCH(h, "prepare_query_kernel");
    return CDTW_OK;
}

}  // namespace cdtw
