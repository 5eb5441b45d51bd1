// z-normalised Euclidean distance of a query to every window of a float64
// series, and its argmin: the GPU-ED path.
//
// Reference: calculate_ed (include/ed.cuh:71-153) zero-pads query and series
// to a multiple of 1e4, runs three cuFFT transforms for the correlation,
// scales it by -2/(sigma*NN) and argsorts all windows with a radix sort,
// printing sqrt(2M + min).  Since sum_k zq_k = 0, the same value is
//   d^2(w) = 2M - 2 * (sum_k zq_k * x_{w+k}) / sigma_w,
// computed here directly in FP64: each thread owns 8 consecutive windows and
// slides them over the query with the window samples in registers (one new
// sample load per query step for 8 FMAs), the query and the series tile staged
// in shared memory (padded one double per eight so the eight-apart thread
// reads do not collide in banks), then an exact FP64 argmin.  No FFT, no sort.
#include "common.cuh"

#include <algorithm>

namespace cdtw {

namespace {

constexpr int kEdThreads = 128;
constexpr int kEdR = 8;                            // windows per thread
constexpr int kEdTile = kEdThreads * kEdR;         // windows per block
constexpr int kEdK = 256;                          // query positions per chunk
constexpr int kEdSpan = kEdTile + kEdK + kEdR;     // samples staged per chunk
constexpr int kEdXs = kEdSpan + (kEdSpan >> 3) + 1;  // with one pad per eight

__device__ __forceinline__ int pad8(int i) { return i + (i >> 3); }

__global__ void __launch_bounds__(kEdThreads)
ed_kernel(const double* __restrict__ x, int64_t N, const double* __restrict__ zq, int M,
          int64_t Nw, const double* __restrict__ sigma, double* __restrict__ out) {
    __shared__ double xs[kEdXs];
    __shared__ double qs[kEdK];
    const int64_t t0 = (int64_t)blockIdx.x * kEdTile;
    const int t = threadIdx.x;
    double acc[kEdR];
#pragma unroll
    for (int r = 0; r < kEdR; ++r) acc[r] = 0.0;
    for (int k0 = 0; k0 < M; k0 += kEdK) {
        const int kn = min(kEdK, M - k0);
        __syncthreads();
        for (int i = t; i < kEdSpan; i += kEdThreads) {
            const int64_t g = t0 + k0 + i;
            xs[pad8(i)] = g < N ? x[g] : 0.0;
        }
        for (int i = t; i < kEdK; i += kEdThreads) qs[i] = i < kn ? zq[k0 + i] : 0.0;
        __syncthreads();
        const int b = t * kEdR;
        double xr[kEdR];
#pragma unroll
        for (int r = 0; r < kEdR; ++r) xr[r] = xs[pad8(b + r)];
        for (int k = 0; k < kn; k += kEdR) {
#pragma unroll
            for (int u = 0; u < kEdR; ++u) {
                const double q = qs[k + u];  // zero beyond kn
#pragma unroll
                for (int r = 0; r < kEdR; ++r) acc[r] = fma(q, xr[(r + u) % kEdR], acc[r]);
                xr[u] = xs[pad8(b + k + u + kEdR)];  // sample b+k+u+R replaces b+k+u
            }
        }
    }
#pragma unroll
    for (int r = 0; r < kEdR; ++r) {
        const int64_t w = t0 + t * kEdR + r;
        if (w < Nw) out[w] = 2.0 * M - 2.0 * acc[r] / sigma[w];
    }
}

__device__ __forceinline__ bool better(double av, long long ai, double bv, long long bi) {
    return av < bv || (av == bv && ai < bi);
}

__global__ void __launch_bounds__(256)
argmin64_kernel(const double* __restrict__ d, int64_t n, ArgMin64* __restrict__ out) {
    __shared__ ArgMin64 red[8];
    double bv = CDTW_INF;
    long long bi = 0x7fffffffffffffffll;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double v = d[i];
        if (better(v, i, bv, bi)) {
            bv = v;
            bi = i;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
        const long long oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (better(ov, oi, bv, bi)) {
            bv = ov;
            bi = oi;
        }
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = ArgMin64{bv, bi};
    __syncthreads();
    if (threadIdx.x == 0) {
        ArgMin64 b = red[0];
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k)
            if (better(red[k].v, red[k].i, b.v, b.i)) b = red[k];
        out[blockIdx.x] = b;
    }
}

__global__ void argmin64_final_kernel(const ArgMin64* __restrict__ p, int n,
                                      ArgMin64* __restrict__ res) {
    __shared__ ArgMin64 red[32];
    ArgMin64 b{CDTW_INF, 0x7fffffffffffffffll};
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        if (better(p[i].v, p[i].i, b.v, b.i)) b = p[i];
    red[threadIdx.x] = b;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)blockDim.x; ++k)
            if (better(red[k].v, red[k].i, b.v, b.i)) b = red[k];
        *res = b;
    }
}

constexpr int kArgminBlocks = 1024;

// z-normalise a float64 query in FP64 (GPU-ed.cu:88 znormalize on the host).
__global__ void __launch_bounds__(256) znorm64_kernel(const double* __restrict__ q, int M,
                                                      double* __restrict__ zq) {
    __shared__ double red[8];
    __shared__ double stat[2];
    const int t = threadIdx.x;
    double s = 0.0;
    for (int i = t; i < M; i += blockDim.x) s += q[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((t & 31) == 0) red[t >> 5] = s;
    __syncthreads();
    if (t == 0) {
        double a = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) a += red[k];
        stat[0] = a / M;
    }
    __syncthreads();
    const double mean = stat[0];
    double v = 0.0;
    for (int i = t; i < M; i += blockDim.x) v = fma(q[i] - mean, q[i] - mean, v);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((t & 31) == 0) red[t >> 5] = v;
    __syncthreads();
    if (t == 0) {
        double a = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) a += red[k];
        const double var = a / M;
        stat[1] = var > 0.0 ? sqrt(var) : 1.0;
    }
    __syncthreads();
    for (int i = t; i < M; i += blockDim.x) zq[i] = (q[i] - mean) / stat[1];
}

}  // namespace

size_t argmin64_partials(int64_t n) { return (size_t)std::min<int64_t>(kArgminBlocks, div_up(n, 256)); }

int launch_argmin64(cdtw_handle h, const double* d, int64_t n, ArgMin64* partial,
                    ArgMin64* res) {
    const int blocks = (int)argmin64_partials(n);
    argmin64_kernel<<<blocks, 256, 0, h->stream>>>(d, n, partial);
    CDTW_LAUNCH(h, "argmin64_kernel");
    argmin64_final_kernel<<<1, 32, 0, h->stream>>>(partial, blocks, res);
    CDTW_LAUNCH(h, "argmin64_final_kernel");
    return CDTW_OK;
}

int launch_znorm64(cdtw_handle h, const double* q, int M, double* zq) {
    znorm64_kernel<<<1, 256, 0, h->stream>>>(q, M, zq);
    CDTW_LAUNCH(h, "znorm64_kernel");
    return CDTW_OK;
}

int launch_ed(cdtw_handle h, const double* x, int64_t N, const double* zq, int M,
              const double* sigma, double* out) {
    const int64_t Nw = N - M + 1;
    ed_kernel<<<(unsigned)div_up(Nw, kEdTile), kEdThreads, 0, h->stream>>>(x, N, zq, M, Nw, sigma,
                                                                          out);
    CDTW_LAUNCH(h, "ed_kernel");
    return CDTW_OK;
}

}  // namespace cdtw
