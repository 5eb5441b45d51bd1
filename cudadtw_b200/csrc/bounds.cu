// Lower bounds of the banded DTW: LB_Kim (the reference's 5x5 front/back
// version), LB_Keogh against the query envelope, and the reverse LB_Keogh of
// the query against the envelope of the data.
//
// Reference: include/bounds.cuh.  register_lb_kim / random_lb_kim
// (bounds.cuh:152-407) run one thread per window with ten uncoalesced stream
// reads each; random_lb_keogh (bounds.cuh:111-144) one thread per listed
// window.  The reverse bound exists only in the UCR Suite
// (UCR_DTW_BIN.cpp:262-282, with the stream envelope of :607).  Here:
//   * lb_kim_kernel: lanes are consecutive windows, so each of the ten sample
//     reads of a warp is one coalesced line; the 5x5 DP runs in registers.
//   * stream_envelope: running min/max over [p-W, p+W] of the stream by the
//     van Herk / Gil-Werman split (prefix and suffix extrema inside segments of
//     2W+1 samples), O(1) work per sample at any W.
//   * lb_keogh_kernel: forward and reverse LB_Keogh of listed windows in one
//     pass over the window (the query envelope and query values are warp-
//     uniform, read once per step for all lanes).
#include "common.cuh"

#include <algorithm>

namespace cdtw {

namespace {

template <bool EU>
__device__ __forceinline__ float lb_kim_window(const float* __restrict__ xw, const Norm& nm,
                                               const float* __restrict__ zq, int M) {
    float sv[10], qv[10];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        sv[k] = znorm(nm, __ldg(xw + k));
        qv[k] = __ldg(zq + k);
        sv[5 + k] = znorm(nm, __ldg(xw + M - 5 + k));
        qv[5 + k] = __ldg(zq + M - 5 + k);
    }
    return lb_kim_dp<EU>(sv, qv);
}

template <bool EU>
__global__ void __launch_bounds__(256)
lb_kim_kernel(const float* __restrict__ x, const double* __restrict__ mu,
              const float* __restrict__ sigma, const float* __restrict__ zq, int M, int Nw,
              const int32_t* __restrict__ idx, int L, float* __restrict__ out,
              unsigned long long* __restrict__ seeds, unsigned* __restrict__ bmax) {
    __shared__ unsigned long long best;
    __shared__ unsigned vmax;
    if (seeds && threadIdx.x == 0) {
        best = ~0ull;
        vmax = 0u;
    }
    if (seeds) __syncthreads();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    float v = CDTW_INF;
    int w = -1;
    if (t < L) {
        w = idx ? idx[t] : t;
        if (w >= 0 && w < Nw) {
            const Norm nm = make_norm(mu[w], sigma[w]);
            v = lb_kim_window<EU>(x + w, nm, zq, M);
        } else {
            v = __int_as_float(0x7fc00000);
        }
        out[t] = v;
    }
    if (seeds) {  // the block's smallest bound: a seed window for the search
        const bool ok = t < L && w >= 0 && w < Nw && v == v;
        const unsigned long long k = warp_min_key(ok, v, (uint32_t)w);
        // and its largest (bounds are >= 0: their bits order as unsigned)
        const unsigned mx = __reduce_max_sync(0xffffffffu, ok ? __float_as_uint(v) : 0u);
        if ((threadIdx.x & 31) == 0) {  // one shared atomic of each kind per warp
            if (k != ~0ull) atomicMin(&best, k);
            atomicMax(&vmax, mx);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            seeds[blockIdx.x] = best;
            bmax[blockIdx.x] = vmax;
        }
    }
}

// Stream envelope of the reverse LB_Keogh (the data envelope of
// UCR_DTW_BIN.cpp:607): env[p] = (min, max) of x over [p-W, p+W] clipped to
// the stream.  One block per tile of T outputs: the tile and its 2W halo are
// staged in shared memory (+inf / -inf outside the stream, which leaves the
// extrema of clipped windows unchanged); spans of 2^j samples are doubled in
// place up to the largest power of two p <= K = 2W+1, and output t takes the
// spans starting at t and at t + K - p.  Coalesced in and out, no scratch.
constexpr int kEnvThreads = 512;
constexpr int kEnvSmemFloats = 50176;  // 196 KB

// PING: two buffers per extremum, one barrier per doubling pass (when they
// fit); otherwise one buffer updated in place in increasing chunks.
template <bool PING>
__global__ void __launch_bounds__(kEnvThreads)
env_window_kernel(const float* __restrict__ x, int64_t N, int W, int T, float2* __restrict__ env,
                  const int* __restrict__ gate, int gate_max) {
    extern __shared__ float esm[];
    if (gate && *(const volatile int*)gate <= gate_max) return;  // not needed by this search
    const int K = 2 * W + 1;
    const int S = T + 2 * W;
    const int64_t ntiles = (N + T - 1) / T;
    // persistent blocks over the tiles (a gated launch costs one wave)
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    float* lo = esm;
    float* hi = esm + S;
    float* lo2 = esm + 2 * S;  // PING only
    float* hi2 = esm + 3 * S;
    const int64_t t0 = tile * T;
    for (int i = threadIdx.x; i < S; i += kEnvThreads) {
        const int64_t g = t0 - W + i;
        const bool in = g >= 0 && g < N;
        const float v = in ? __ldg(x + g) : 0.f;
        lo[i] = in ? v : CDTW_INF;
        hi[i] = in ? v : -CDTW_INF;
    }
    __syncthreads();
    int p = 1;
    for (; 2 * p <= K; p *= 2) {
        // entry i becomes the extremum of [i, i + 2p)
        if (PING) {
            for (int i = threadIdx.x; i < S; i += kEnvThreads) {
                const int j = min(i + p, S - 1);
                lo2[i] = fminf(lo[i], lo[j]);
                hi2[i] = fmaxf(hi[i], hi[j]);
            }
            __syncthreads();
            float* t = lo;
            lo = lo2;
            lo2 = t;
            t = hi;
            hi = hi2;
            hi2 = t;
        } else {
            // chunks in increasing i, so a partner i + p > i is never one this
            // pass already rewrote
            for (int i0 = 0; i0 < S - p; i0 += kEnvThreads) {
                const int i = i0 + threadIdx.x;
                float a = 0.f, b = 0.f;
                if (i < S - p) {
                    a = fminf(lo[i], lo[i + p]);
                    b = fmaxf(hi[i], hi[i + p]);
                }
                __syncthreads();
                if (i < S - p) {
                    lo[i] = a;
                    hi[i] = b;
                }
                __syncthreads();
            }
        }
    }
    for (int t = threadIdx.x; t < T; t += kEnvThreads) {
        if (t0 + t >= N) break;
        const int c = t + K - p;
        env[t0 + t] = make_float2(fminf(lo[t], lo[c]), fmaxf(hi[t], hi[c]));
    }
    __syncthreads();  // the next tile restages the buffers
    }
}

// Forward LB_Keogh (window vs query envelope, bounds.cuh:128-140) and reverse
// LB_Keogh (query vs data envelope, UCR_DTW_BIN.cpp:262-282) of listed windows.
template <bool EU>
__global__ void __launch_bounds__(256)
lb_keogh_kernel(const float* __restrict__ x, const double* __restrict__ mu,
                const float* __restrict__ sigma, const float* __restrict__ zq,
                const float2* __restrict__ qenv, const float2* __restrict__ xenv, int M, int Nw,
                const int32_t* __restrict__ idx, int L, float* __restrict__ fwd,
                float* __restrict__ rev) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= L) return;
    const int w = idx ? idx[t] : t;
    if (w < 0 || w >= Nw) {
        if (fwd) fwd[t] = __int_as_float(0x7fc00000);
        if (rev) rev[t] = __int_as_float(0x7fc00000);
        return;
    }
    const Norm nm = make_norm(mu[w], sigma[w]);
    float af = 0.f, ar = 0.f;
    for (int k = 0; k < M; ++k) {
        const float z = znorm(nm, __ldg(x + w + k));
        const float2 e = __ldg(qenv + k);
        const float df = max3f(z - e.y, e.x - z, 0.f);
        af = EU ? fmaf(df, df, af) : af + df;
        if (rev) {
            const float2 d = __ldg(xenv + w + k);
            const float q = __ldg(zq + k);
            const float dr = max3f(q - znorm(nm, d.y), znorm(nm, d.x) - q, 0.f);
            ar = EU ? fmaf(dr, dr, ar) : ar + dr;
        }
    }
    if (fwd) fwd[t] = af;
    if (rev) rev[t] = ar;
}

// LB_Kim of every window for the search's first pass, with per block of
// kKimSeedBlock windows the one of smallest bound (a seed) and the largest
// bound.  A warp takes one such block, a lane eight consecutive windows:
// their front samples are twelve consecutive stream values, their back
// samples another twelve, and the ten query values stay in registers (the
// same arithmetic as lb_kim_kernel, window by window).  Away from the stream's
// end and with 16-byte aligned inputs a lane loads them as vectors: its eight
// means as four double2, sigmas as two float4, front samples as three float4
// and back samples as four aligned float4 shifted by (M - 5) mod 4 (13 loads
// against 40 scalar ones, whose lane strides spread each instruction over 8 to
// 16 cache lines).
constexpr int kKimSeedBlock = 256;
constexpr int kKimPerLane = kKimSeedBlock / 32;

template <bool EU, int SH>  // SH = (M - 5) mod 4
__global__ void __launch_bounds__(256)
lb_kim_all_kernel(const float* __restrict__ x, int64_t N, const double* __restrict__ mu,
                  const float* __restrict__ sigma, const float* __restrict__ zq, int M, int Nw,
                  float* __restrict__ out, unsigned long long* __restrict__ seeds,
                  unsigned* __restrict__ bmax) {
    float qf[5], qb[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        qf[k] = __ldg(zq + k);
        qb[k] = __ldg(zq + M - 5 + k);
    }
    const int lane = threadIdx.x & 31;
    const bool vec = ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(mu) |
                       reinterpret_cast<uintptr_t>(sigma)) & 15) == 0;
    const int64_t nblk = ((int64_t)Nw + kKimSeedBlock - 1) / kKimSeedBlock;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t b = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < nblk;
         b += nwarps) {
        const int64_t w0 = b * kKimSeedBlock + (int64_t)lane * kKimPerLane;
        unsigned long long best = ~0ull;
        unsigned mx = 0u;
        if (w0 < Nw) {
            float xf[kKimPerLane + 4], xb[kKimPerLane + 4];
            double mv[kKimPerLane];
            float sv[kKimPerLane];
            const int64_t ab = w0 + M - 5 - SH;  // first back float4 (w0 is a multiple of 8)
            if (vec && w0 + kKimPerLane <= Nw && ab + 16 <= N) {
                const double2* m2 = reinterpret_cast<const double2*>(mu + w0);
                const float4* s4 = reinterpret_cast<const float4*>(sigma + w0);
                const float4* f4 = reinterpret_cast<const float4*>(x + w0);
                const float4* b4 = reinterpret_cast<const float4*>(x + ab);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const double2 d = __ldg(m2 + j);
                    mv[2 * j] = d.x;
                    mv[2 * j + 1] = d.y;
                }
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const float4 v = __ldg(s4 + j);
                    sv[4 * j] = v.x;
                    sv[4 * j + 1] = v.y;
                    sv[4 * j + 2] = v.z;
                    sv[4 * j + 3] = v.w;
                }
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const float4 v = __ldg(f4 + j);
                    xf[4 * j] = v.x;
                    xf[4 * j + 1] = v.y;
                    xf[4 * j + 2] = v.z;
                    xf[4 * j + 3] = v.w;
                }
                float bv[16];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const float4 v = __ldg(b4 + j);
                    bv[4 * j] = v.x;
                    bv[4 * j + 1] = v.y;
                    bv[4 * j + 2] = v.z;
                    bv[4 * j + 3] = v.w;
                }
#pragma unroll
                for (int j = 0; j < kKimPerLane + 4; ++j) xb[j] = bv[SH + j];
            } else {
#pragma unroll
                for (int j = 0; j < kKimPerLane + 4; ++j) {
                    xf[j] = (w0 + j < N) ? __ldg(x + w0 + j) : 0.f;
                    xb[j] = (w0 + M - 5 + j < N) ? __ldg(x + w0 + M - 5 + j) : 0.f;
                }
#pragma unroll
                for (int i = 0; i < kKimPerLane; ++i) {
                    const int64_t w = min(w0 + i, (int64_t)Nw - 1);
                    mv[i] = __ldg(mu + w);
                    sv[i] = __ldg(sigma + w);
                }
            }
            float f[kKimPerLane];
#pragma unroll
            for (int i = 0; i < kKimPerLane; ++i) {
                const int64_t w = w0 + i;
                f[i] = CDTW_INF;
                if (w < Nw) {
                    const Norm nm = make_norm(mv[i], sv[i]);
                    float sf[5], sb[5];
#pragma unroll
                    for (int k = 0; k < 5; ++k) {
                        sf[k] = znorm(nm, xf[i + k]);
                        sb[k] = znorm(nm, xb[i + k]);
                    }
                    f[i] = lb_kim_front<EU>(sf, qf) + lb_kim_back<EU>(sb, qb);
                    if (f[i] == f[i]) {
                        best = min(best, pack_key(f[i], (uint32_t)w));
                        mx = max(mx, __float_as_uint(f[i]));
                    }
                }
            }
            if (w0 + kKimPerLane <= Nw) {  // out is 256-byte aligned, w0 a multiple of 8
                float4* o = reinterpret_cast<float4*>(out + w0);
                o[0] = make_float4(f[0], f[1], f[2], f[3]);
                o[1] = make_float4(f[4], f[5], f[6], f[7]);
            } else {
#pragma unroll
                for (int i = 0; i < kKimPerLane; ++i)
                    if (w0 + i < Nw) out[w0 + i] = f[i];
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) best = min(best, __shfl_xor_sync(0xffffffffu, best, o));
        mx = __reduce_max_sync(0xffffffffu, mx);
        if (lane == 0) {
            seeds[b] = best;
            bmax[b] = mx;
        }
    }
}

}  // namespace

int launch_lb_kim_all(cdtw_handle h, const float* x, int64_t N, const double* mu,
                      const float* sigma, bool euclid, float* out, unsigned long long* seeds,
                      unsigned* bmax) {
    const QueryPack& q = h->q;
    if (q.M < 11)
        return set_error(h, CDTW_EINVAL,
                         "LB_Kim is a 10-point DTW: the query needs at least 11 samples");
    const int64_t Nw = N - q.M + 1;
    if (Nw <= 0) return CDTW_OK;
    const int64_t warps = div_up(Nw, kKimSeedBlock);
    const unsigned blocks = (unsigned)std::max<int64_t>(
        1, std::min<int64_t>(div_up(warps, 8), (int64_t)h->sm_count * 8));
    using KimAll = void (*)(const float*, int64_t, const double*, const float*, const float*, int,
                            int, float*, unsigned long long*, unsigned*);
    static const KimAll eu[4] = {lb_kim_all_kernel<true, 0>, lb_kim_all_kernel<true, 1>,
                                 lb_kim_all_kernel<true, 2>, lb_kim_all_kernel<true, 3>};
    static const KimAll mh[4] = {lb_kim_all_kernel<false, 0>, lb_kim_all_kernel<false, 1>,
                                 lb_kim_all_kernel<false, 2>, lb_kim_all_kernel<false, 3>};
    const KimAll k = (euclid ? eu : mh)[(q.M - 5) & 3];
    k<<<blocks, 256, 0, h->stream>>>(x, N, mu, sigma, q.zq, q.M, (int)Nw, out, seeds, bmax);
    CDTW_LAUNCH(h, "lb_kim_all_kernel");
    return CDTW_OK;
}

int launch_lb_kim(cdtw_handle h, const float* x, int64_t N, const double* mu, const float* sigma,
                  const int32_t* idx, int64_t L, bool euclid, float* out,
                  unsigned long long* seeds, unsigned* bmax) {
    const QueryPack& q = h->q;
    if (q.M < 11)
        return set_error(h, CDTW_EINVAL,
                         "LB_Kim is a 10-point DTW: the query needs at least 11 samples");
    if (L <= 0) return CDTW_OK;
    const int Nw = (int)(N - q.M + 1);
    const unsigned blocks = (unsigned)div_up(L, 256);
    if (euclid)
        lb_kim_kernel<true><<<blocks, 256, 0, h->stream>>>(x, mu, sigma, q.zq, q.M, Nw, idx,
                                                            (int)L, out, seeds, bmax);
    else
        lb_kim_kernel<false><<<blocks, 256, 0, h->stream>>>(x, mu, sigma, q.zq, q.M, Nw, idx,
                                                             (int)L, out, seeds, bmax);
    CDTW_LAUNCH(h, "lb_kim_kernel");
    return CDTW_OK;
}

size_t stream_envelope_scratch_bytes(int64_t) { return 0; }

int launch_stream_envelope(cdtw_handle h, const float* x, int64_t N, int W, float*,
                           float2* env, const int* gate, int gate_max) {
    // tile: at least 2048 outputs (or 2W when the halo is larger); four
    // arrays (ping-pong) when they fit the shared-memory budget, else two
    if (kEnvSmemFloats / 2 - 2 * W < 1)
        return set_error(h, CDTW_EUNSUPPORTED, "band W=%d too wide for the stream envelope", W);
    const bool ping = kEnvSmemFloats / 4 - 2 * W >= 2048;
    const int arrays = ping ? 4 : 2;
    const int T = std::max(1, std::min(std::max(2048, 2 * W), kEnvSmemFloats / arrays - 2 * W));
    const size_t smem = (size_t)arrays * (T + 2 * W) * sizeof(float);
    const void* k = ping ? (const void*)env_window_kernel<true> : (const void*)env_window_kernel<false>;
    CDTW_CUDA(h, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    CDTW_CUDA(h, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kEnvThreads, smem));
    const unsigned grid = (unsigned)std::max<int64_t>(
        1, std::min<int64_t>(div_up(N, T), (int64_t)std::max(per_sm, 1) * h->sm_count));
    if (ping)
        env_window_kernel<true><<<grid, kEnvThreads, smem, h->stream>>>(x, N, W, T, env, gate,
                                                                       gate_max);
    else
        env_window_kernel<false><<<grid, kEnvThreads, smem, h->stream>>>(x, N, W, T, env, gate,
                                                                        gate_max);
    CDTW_LAUNCH(h, "env_window_kernel");
    return CDTW_OK;
}

int launch_lb_keogh(cdtw_handle h, const float* x, int64_t N, const double* mu,
                    const float* sigma, const float2* xenv, const int32_t* idx, int64_t L,
                    bool euclid, float* fwd, float* rev) {
    const QueryPack& q = h->q;
    if (L <= 0) return CDTW_OK;
    const int Nw = (int)(N - q.M + 1);
    const unsigned blocks = (unsigned)div_up(L, 256);
    if (euclid)
        lb_keogh_kernel<true><<<blocks, 256, 0, h->stream>>>(x, mu, sigma, q.zq, q.env, xenv,
                                                              q.M, Nw, idx, (int)L, fwd, rev);
    else
        lb_keogh_kernel<false><<<blocks, 256, 0, h->stream>>>(x, mu, sigma, q.zq, q.env, xenv,
                                                               q.M, Nw, idx, (int)L, fwd, rev);
    CDTW_LAUNCH(h, "lb_keogh_kernel");
    return CDTW_OK;
}

}  // namespace cdtw
