// Greedy locally-optimal warping path inside the Sakoe-Chiba band (LDTW),
// z-normalised, for every window: the GPU-LDTW path.
//
// Reference: ztsh2_ldtw (include/ldtw.cuh:294-391) and its serial twin
// z_serial_ldtw (ldtw.cuh:74-127): one path of at most 2M-2 steps per window;
// at (i, j) take the diagonal if it is strictly cheaper than both the cell
// below and the cell to the right, else "down" if the diagonal is not cheaper
// than it and it is cheaper than "right", else "right"; moves outside the
// matrix or the band cost INFTY = 1e10 (ldtw.cuh:8).  One thread per window
// here too (a path is inherently sequential), in FP64 so the branch decisions
// match the FP64 oracle; the four values a step reads (two query, two window
// samples) are carried in registers and only the entering ones are loaded.
#include "common.cuh"

#include <algorithm>

namespace cdtw {

namespace {

template <bool EU>
__device__ __forceinline__ double lcost(double d) { return EU ? d * d : fabs(d); }

template <bool EU>
__global__ void __launch_bounds__(128)
ldtw_kernel(const float* __restrict__ x, const double* __restrict__ mu,
            const double* __restrict__ sigma, const double* __restrict__ zq, int M, int W,
            int64_t Nw, double* __restrict__ out) {
    const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= Nw) return;
    const double INFTY = 1e10;
    const double m = mu[w], s = sigma[w];
    const float* __restrict__ xw = x + w;
    int i = 0, j = 0;
    double q0 = zq[0], q1 = (M > 1) ? zq[1] : 0.0;
    double s0 = ((double)xw[0] - m) / s, s1 = (M > 1) ? ((double)xw[1] - m) / s : 0.0;
    double d = lcost<EU>(q0 - s0);
    // every step advances i or j, so 2M-2 steps reach (M-1, M-1); the cap only
    // guards against non-finite input
    for (int it = 0; it < 2 * M && (i + 1 != M || j + 1 != M); ++it) {
        double diag = INFTY, rght = INFTY, down = INFTY;
        if (i + 1 < M && j + 1 < M) diag = lcost<EU>(q1 - s1);
        if (i + 1 < M && abs(i - j + 1) <= W) down = lcost<EU>(q1 - s0);
        if (j + 1 < M && abs(j - i + 1) <= W) rght = lcost<EU>(q0 - s1);
        const bool diagSdown = diag < down, diagSrght = diag < rght, downSrght = down < rght;
        bool mi, mj;
        if (diagSdown && diagSrght) {
            d += diag;
            mi = mj = true;
        } else if (!diagSdown && downSrght) {
            d += down;
            mi = true;
            mj = false;
        } else {
            d += rght;
            mi = false;
            mj = true;
        }
        if (mi) {
            ++i;
            q0 = q1;
            q1 = (i + 1 < M) ? zq[i + 1] : 0.0;
        }
        if (mj) {
            ++j;
            s0 = s1;
            s1 = (j + 1 < M) ? ((double)xw[j + 1] - m) / s : 0.0;
        }
    }
    out[w] = d;
}

// The reference's own FP32 arithmetic, for drop-in index parity with its
// GPU-LDTW.  The query is z-normalised as the reference driver does on the
// host (znormalize, stats.cuh:8-28: float sums in order, population sigma,
// (x - avg) / std), by one thread, without fused multiply-adds.
__global__ void ldtw_ref_query_kernel(const float* __restrict__ qraw, int M,
                                      float* __restrict__ zq) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    float avg = 0.f, sd = 0.f;
    for (int i = 0; i < M; ++i) avg = __fadd_rn(avg, qraw[i]);
    avg = __fdiv_rn(avg, (float)M);
    for (int i = 0; i < M; ++i) sd = __fadd_rn(sd, __fmul_rn(qraw[i], qraw[i]));
    sd = __fsqrt_rn(__fsub_rn(__fdiv_rn(sd, (float)M), __fmul_rn(avg, avg)));
    for (int i = 0; i < M; ++i) zq[i] = __fdiv_rn(__fsub_rn(qraw[i], avg), sd);
}

template <bool EU>
__device__ __forceinline__ float lcost_ref(float d) {
    return EU ? __fmul_rn(d, d) : fabsf(d);
}

// One window per thread, the steps of ztsh2_ldtw (ZN) / tsh2_ldtw
// (ldtw.cuh:294-391 / :199-291) in FP32: exactly 2M-2 relaxations, moves
// out of the matrix or the band cost INFTY = 1e10, the tie rule of
// ldtw.cuh:368-383, and nothing added once (M-1, M-1) is reached.  ZN: the
// window statistics of avg_std<double> (stats.cuh:30-52): the window mean of
// x and of x^2 in FP64 rounded to float, variance E[x^2] - mu^2 in float
// (the fused multiply-add nvcc makes of stats.cuh:49), sigma = 1 where it is
// not positive; samples normalised as (s - avg) / std in float.  (The
// reference takes the window sums as differences of FP64 prefix sums; here
// they are summed directly, equal to a few FP64 ulps.)
template <bool EU, bool ZN>
__global__ void __launch_bounds__(128)
ldtw_ref_kernel(const float* __restrict__ x, const float* __restrict__ zq, int M, int W,
                int64_t Nw, float* __restrict__ out) {
    const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= Nw) return;
    const float INFTY = 1e10f;
    const float* __restrict__ xw = x + w;
    float avg = 0.f, sd = 1.f;
    if (ZN) {
        double s1 = 0.0, s2 = 0.0;
        for (int k = 0; k < M; ++k) {
            const double v = (double)__ldg(xw + k);
            s1 += v;
            s2 += v * v;
        }
        avg = (float)(s1 / M);
        const float ex2 = (float)(s2 / M);
        const float var = __fmaf_rn(-avg, avg, ex2);
        sd = var > 0.f ? __fsqrt_rn(var) : 1.f;
    }
    auto sp = [&](int j) {
        const float v = __ldg(xw + j);
        return ZN ? __fdiv_rn(__fsub_rn(v, avg), sd) : v;
    };
    float d = lcost_ref<EU>(__fsub_rn(zq[0], sp(0)));
    int i = 0, j = 0;
    for (int k = 0; k < 2 * M - 2; ++k) {
        const bool vi = i + 1 < M, vj = j + 1 < M;
        const bool cd = abs(i - j + 1) <= W, cr = abs(j - i + 1) <= W;
        const float sp0 = sp(j), sp1 = sp(vj ? j + 1 : j);
        const float qp0 = zq[i], qp1 = zq[vi ? i + 1 : i];
        const float diag = (vi && vj) ? lcost_ref<EU>(__fsub_rn(qp1, sp1)) : INFTY;
        const float down = (vi && cd) ? lcost_ref<EU>(__fsub_rn(qp1, sp0)) : INFTY;
        const float rght = (vj && cr) ? lcost_ref<EU>(__fsub_rn(qp0, sp1)) : INFTY;
        const bool diagSdown = diag < down, diagSrght = diag < rght, downSrght = down < rght;
        float bsf;
        if (diagSdown && diagSrght) {
            bsf = diag;
            i = min(i + 1, M - 1);
            j = min(j + 1, M - 1);
        } else if (!diagSdown && downSrght) {
            bsf = down;
            i = min(i + 1, M - 1);
        } else {
            bsf = rght;
            j = min(j + 1, M - 1);
        }
        d = __fadd_rn(d, (vi || vj) ? bsf : 0.f);
    }
    out[w] = d;
}

// Packed (float bits, index) minimum; values are >= 0, so their bits order as
// unsigned ints, and ties keep the lowest index (determine_min's first strict
// minimum, ldtw.cuh:177-192).
__global__ void argmin_f32_kernel(const float* __restrict__ v, int64_t n,
                                  unsigned long long* __restrict__ key) {
    unsigned long long best = ~0ull;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float a = v[i];
        if (a == a) best = min(best, pack_key(a, (uint32_t)i));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = min(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0 && best != ~0ull) atomicMin(key, best);
}

}  // namespace

int launch_ldtw_ref(cdtw_handle h, const float* x, int64_t N, bool euclid, bool znorm,
                    float* qwork, float* out) {
    const QueryPack& q = h->q;
    if (!q.qraw) return set_error(h, CDTW_EINVAL, "query pack without the raw query");
    const int64_t Nw = N - q.M + 1;
    const float* zq = q.qraw;
    if (znorm) {
        ldtw_ref_query_kernel<<<1, 32, 0, h->stream>>>(q.qraw, q.M, qwork);
        CDTW_LAUNCH(h, "ldtw_ref_query_kernel");
        zq = qwork;
    }
    const unsigned blocks = (unsigned)div_up(Nw, 128);
    auto k = euclid ? (znorm ? ldtw_ref_kernel<true, true> : ldtw_ref_kernel<true, false>)
                    : (znorm ? ldtw_ref_kernel<false, true> : ldtw_ref_kernel<false, false>);
    k<<<blocks, 128, 0, h->stream>>>(x, zq, q.M, q.W, Nw, out);
    CDTW_LAUNCH(h, "ldtw_ref_kernel");
    return CDTW_OK;
}

int launch_argmin_f32(cdtw_handle h, const float* v, int64_t n, unsigned long long* key) {
    const unsigned blocks = (unsigned)std::max<int64_t>(
        1, std::min<int64_t>(div_up(n, 256), (int64_t)h->sm_count * 8));
    argmin_f32_kernel<<<blocks, 256, 0, h->stream>>>(v, n, key);
    CDTW_LAUNCH(h, "argmin_f32_kernel");
    return CDTW_OK;
}

int launch_ldtw(cdtw_handle h, const float* x, int64_t N, const double* mu, const double* sigma,
                bool euclid, double* out) {
    const QueryPack& q = h->q;
    const int64_t Nw = N - q.M + 1;
    const unsigned blocks = (unsigned)div_up(Nw, 128);
    if (euclid)
        ldtw_kernel<true><<<blocks, 128, 0, h->stream>>>(x, mu, sigma, q.zq64, q.M, q.W, Nw, out);
    else
        ldtw_kernel<false><<<blocks, 128, 0, h->stream>>>(x, mu, sigma, q.zq64, q.M, q.W, Nw, out);
    CDTW_LAUNCH(h, "ldtw_kernel");
    return CDTW_OK;
}

}  // namespace cdtw
