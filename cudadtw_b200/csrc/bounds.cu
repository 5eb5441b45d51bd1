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
              unsigned long long* __restrict__ seeds) {
    __shared__ unsigned long long best;
    if (seeds && threadIdx.x == 0) best = ~0ull;
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
        if (t < L && w >= 0 && w < Nw && v == v) atomicMin(&best, pack_key(v, (uint32_t)w));
        __syncthreads();
        if (threadIdx.x == 0) seeds[blockIdx.x] = best;
    }
}

// van Herk / Gil-Werman, pass 1: prefix and suffix min/max inside segments
// of K = 2W+1 samples (one thread per segment).
__global__ void __launch_bounds__(128)
env_segments_kernel(const float* __restrict__ x, int64_t N, int K, float* __restrict__ pmin,
                    float* __restrict__ pmax, float* __restrict__ smin, float* __restrict__ smax) {
    const int64_t seg = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t a = seg * K;
    if (a >= N) return;
    const int64_t b = min(a + K, N);
    float lo = CDTW_INF, hi = -CDTW_INF;
    for (int64_t i = a; i < b; ++i) {
        const float v = x[i];
        lo = fminf(lo, v);
        hi = fmaxf(hi, v);
        pmin[i] = lo;
        pmax[i] = hi;
    }
    lo = CDTW_INF;
    hi = -CDTW_INF;
    for (int64_t i = b - 1; i >= a; --i) {
        const float v = x[i];
        lo = fminf(lo, v);
        hi = fmaxf(hi, v);
        smin[i] = lo;
        smax[i] = hi;
    }
}

// pass 2: extrema over [p-W, p+W] clipped to the stream.  A full window of
// K samples either starts a segment (prefix extremum at its end) or spans two
// segments (suffix extremum at its start combined with the prefix extremum
// at its end); windows clipped at the stream ends are handled the same way.
__global__ void __launch_bounds__(256)
env_combine_kernel(const float* __restrict__ x, int64_t N, int W, const float* __restrict__ pmin,
                   const float* __restrict__ pmax, const float* __restrict__ smin,
                   const float* __restrict__ smax, float2* __restrict__ env) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    const int64_t K = 2 * (int64_t)W + 1;
    const int64_t a = max((int64_t)0, p - W), b = min(N - 1, p + W);
    const int64_t sa = a / K, sb = b / K;
    float lo, hi;
    if (sa != sb) {
        lo = fminf(smin[a], pmin[b]);
        hi = fmaxf(smax[a], pmax[b]);
    } else if (a == sa * K) {  // window starts its segment
        lo = pmin[b];
        hi = pmax[b];
    } else if (b == min(N, (sa + 1) * K) - 1) {  // window ends its segment
        lo = smin[a];
        hi = smax[a];
    } else {  // clipped on both sides (stream shorter than the band): direct
        lo = CDTW_INF;
        hi = -CDTW_INF;
        for (int64_t i = a; i <= b; ++i) {
            lo = fminf(lo, x[i]);
            hi = fmaxf(hi, x[i]);
        }
    }
    env[p] = make_float2(lo, hi);
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

}  // namespace

int launch_lb_kim(cdtw_handle h, const float* x, int64_t N, const double* mu, const float* sigma,
                  const int32_t* idx, int64_t L, bool euclid, float* out,
                  unsigned long long* seeds) {
    const QueryPack& q = h->q;
    if (q.M < 11)
        return set_error(h, CDTW_EINVAL,
                         "LB_Kim is a 10-point DTW: the query needs at least 11 samples");
    if (L <= 0) return CDTW_OK;
    const int Nw = (int)(N - q.M + 1);
    const unsigned blocks = (unsigned)div_up(L, 256);
    if (euclid)
        lb_kim_kernel<true><<<blocks, 256, 0, h->stream>>>(x, mu, sigma, q.zq, q.M, Nw, idx,
                                                            (int)L, out, seeds);
    else
        lb_kim_kernel<false><<<blocks, 256, 0, h->stream>>>(x, mu, sigma, q.zq, q.M, Nw, idx,
                                                             (int)L, out, seeds);
    CDTW_LAUNCH(h, "lb_kim_kernel");
    return CDTW_OK;
}

size_t stream_envelope_scratch_bytes(int64_t N) { return (size_t)N * 4 * sizeof(float); }

int launch_stream_envelope(cdtw_handle h, const float* x, int64_t N, int W, float* scratch,
                           float2* env) {
    const int K = 2 * W + 1;
    float* pmin = scratch;
    float* pmax = scratch + N;
    float* smin = scratch + 2 * N;
    float* smax = scratch + 3 * N;
    const int64_t segs = div_up(N, K);
    env_segments_kernel<<<(unsigned)div_up(segs, 128), 128, 0, h->stream>>>(x, N, K, pmin, pmax,
                                                                          smin, smax);
    CDTW_LAUNCH(h, "env_segments_kernel");
    env_combine_kernel<<<(unsigned)div_up(N, 256), 256, 0, h->stream>>>(x, N, W, pmin, pmax,
                                                                      smin, smax, env);
    CDTW_LAUNCH(h, "env_combine_kernel");
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
