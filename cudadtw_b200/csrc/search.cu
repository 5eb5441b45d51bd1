// Pruned subsequence search: the replacement of prune_cdtw
// (include/cdtw.cuh:510-592).
//
// The reference sorts LB_Kim of all windows (a full radix sort), runs the
// cDTW of the first chunk, then loops on the host over doubling chunks with
// LB_Keogh -> threshold compaction -> cDTW -> min-reduce, with cudaMalloc/
// cudaFree and two or three blocking device-to-host reads per chunk.  Here the
// whole search is one fixed sequence of launches on the handle's stream with
// a single device-to-host read of the result at the end:
//
//   1. LB_Kim of every window; each block also records its smallest bound
//      (a seed window).
//   2. cDTW of the seed windows -> first best-so-far, a packed
//      (distance, window) key updated by atomicMin.
//   3. Compaction of the windows whose LB_Kim is below the best-so-far.
//   4. Forward LB_Keogh (query envelope) and reverse LB_Keogh (data
//      envelope, as UCR_DTW_BIN.cpp:262-282) of those, abandoned once the
//      bound passed the best-so-far; survivors keep their best bound and
//      their forward LB_Keogh.  Few, scattered survivors: a warp per window
//      with the window's own envelope; many: the envelope of the whole stream
//      and a thread per window (the count is read on the device).
//   5. cDTW of the survivors with early abandoning against the live
//      best-so-far, folded into the key: as pairwise wavefronts when few and
//      long, else by the register-band (W <= 96) or lane-group kernels.
// No sort, no host loop; graph-capturable launch sequence.
#include "common.cuh"

#include <algorithm>
#include <set>
#include <vector>

namespace cdtw {

namespace {

struct SearchWs {
    float* lbkim = nullptr;
    unsigned long long* seeds = nullptr;
    unsigned* bmax = nullptr;  // largest LB_Kim of each block (float bits)
    Cand* seed_cands = nullptr;
    int* q1 = nullptr;
    Cand* q2 = nullptr;
    float2* xenv = nullptr;
    float* envscratch = nullptr;
    // [0] n1, [1] n2, [2] work seeds, [3] work main, [4] n seeds, [5] largest LB_Kim (bits)
    int* ctr = nullptr;
    unsigned long long* key = nullptr;
    float* seed_z = nullptr;  // z-normalised seed windows (seed_cap floats)
    float* seed_d = nullptr;  // their cDTW (max(kSeedMax, kWaveSurvivors) floats)
    int64_t seed_cap = 0;
};

constexpr int kKimBlock = 256;
constexpr int kSeedMax = 4096;                     // seed_target's upper limit
constexpr int64_t kSeedZMax = (int64_t)1 << 24;    // floats of seed windows (64 MB)
constexpr float kSeedBoundSlack = 1.0f + 1e-4f;
constexpr int kWaveSurvivors = 8192;               // survivors cDTW'd as wavefronts (at most)
constexpr int kWaveFew = 256;                      // of them, run by the widest lane groups
constexpr double kWaveMinCells = 4.0e4;            // band cells per window for that

// The seed windows, z-normalised (FP64 arithmetic, rounded once), one row of
// M floats per seed: the subjects of the seeds' pairwise cDTW.  One warp per
// seed.
__global__ void seed_gather_kernel(const float* __restrict__ x, const double* __restrict__ mu,
                                   const float* __restrict__ sigma, const Cand* __restrict__ cands,
                                   int nseed, int M, float* __restrict__ z) {
    const int lane = threadIdx.x & 31;
    const int i = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (i >= nseed) return;
    const int w = cands[i].w;
    const double m = mu[w], inv = 1.0 / (double)sigma[w];
    float* zi = z + (int64_t)i * M;
    for (int j = lane; j < M; j += 32) zi[j] = (float)(((double)__ldg(x + w + j) - m) * inv);
}

// The survivors of the bounds when there are at most `cap`, z-normalised
// exactly as the search kernels do (make_norm / znorm), for their pairwise
// wavefront cDTW (which runs the first *count rows only).  Thread 0 starts
// the search kernels' work counter at cap (they then find nothing left), or
// at 0 when there are more survivors than cap (the wavefront pass is skipped
// and they take all).
__global__ void wave_gather_kernel(const float* __restrict__ x, const double* __restrict__ mu,
                                   const float* __restrict__ sigma, const Cand* __restrict__ cands,
                                   const int* __restrict__ count, int cap, int M,
                                   float* __restrict__ z, int* __restrict__ work) {
    const int lane = threadIdx.x & 31;
    const int i = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int n = *count;
    if (blockIdx.x == 0 && threadIdx.x == 0) *work = n > cap ? 0 : cap;
    if (i >= n || n > cap) return;
    const int w = cands[i].w;
    const Norm nm = make_norm(mu[w], sigma[w]);
    float* zi = z + (int64_t)i * M;
    for (int j = lane; j < M; j += 32) zi[j] = znorm(nm, __ldg(x + w + j));
}

// Exact keys of the wavefront survivors: (distance, window) into the packed
// best-so-far, as the search kernels would (their cells and z-values are the
// same, so the distances are bit-identical).
__global__ void wave_keys_kernel(const float* __restrict__ d, const Cand* __restrict__ cands,
                                 const int* __restrict__ count, int cap,
                                 unsigned long long* __restrict__ key) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = *count > cap ? 0 : *count;
    const bool ok = i < n && d[i] == d[i] && d[i] < CDTW_INF;
    const unsigned long long k =
        warp_min_key(ok, ok ? d[i] : CDTW_INF, ok ? (uint32_t)cands[i].w : 0xffffffffu);
    if ((threadIdx.x & 31) == 0 && k != ~0ull) atomicMin(key, k);
}

// First best-so-far from the seeds' cDTW: the smallest distance, raised by
// kSeedBoundSlack relative and 1e-6 per query sample absolute, and paired with
// no window (index 0xffffffff).  The seed z-values are rounded once from FP64,
// the search kernels' differ by a few ulps at most, so the seed window's own
// distance as the search kernels compute it lies below this bound (also for
// an exact match, distance 0): the bound prunes nothing that could be the
// best, and the best window replaces it in the key.
__global__ void seed_bound_kernel(const float* __restrict__ d, const Cand* __restrict__ cands,
                                  int nseed, int M, unsigned long long* __restrict__ key) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool ok = i < nseed && cands[i].lb < CDTW_INF && d[i] == d[i] && d[i] < CDTW_INF;
    const float b = ok ? d[i] * kSeedBoundSlack + 1e-6f * (float)M : CDTW_INF;
    const unsigned long long k = warp_min_key(ok, b, 0xffffffffu);
    if ((threadIdx.x & 31) == 0 && k != ~0ull) atomicMin(key, k);
}

// The same raising for seeds whose cDTW the search kernels computed into a
// key of their own (skey: the best seed's packed distance and window).
__global__ void seed_key_bound_kernel(const unsigned long long* __restrict__ skey, int M,
                                      unsigned long long* __restrict__ key) {
    const unsigned long long k = *skey;
    if (k == ~0ull) return;
    const float d = key_dist(k);
    if (!(d < CDTW_INF)) return;
    atomicMin(key, pack_key(d * kSeedBoundSlack + 1e-6f * (float)M, 0xffffffffu));
}

// Seed candidates: the smallest-bound window of each group of G blocks; with
// bmax, the largest LB_Kim of all windows into *kmax (float bits).
__global__ void seeds_to_cands_kernel(const unsigned long long* __restrict__ seeds,
                                      const unsigned* __restrict__ bmax, int nblk, int G,
                                      Cand* __restrict__ cands, int* __restrict__ nseeds,
                                      unsigned* __restrict__ kmax) {
    // a warp per group of G blocks (groups of hundreds of blocks are common)
    const int lane = threadIdx.x & 31;
    const int i = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int n = (nblk + G - 1) / G;
    if (i == 0 && lane == 0) *nseeds = n;
    if (i >= n) return;  // whole warps
    unsigned long long k = ~0ull;
    unsigned mx = 0u;
    for (int b = i * G + lane; b < min(nblk, (i + 1) * G); b += 32) {
        k = min(k, seeds[b]);
        if (bmax) mx = max(mx, bmax[b]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) k = min(k, __shfl_xor_sync(0xffffffffu, k, o));
    mx = __reduce_max_sync(0xffffffffu, mx);
    if (lane != 0) return;
    if (mx) atomicMax(kmax, mx);
    Cand c;
    c.w = (k == ~0ull) ? 0 : (int)(uint32_t)k;
    c.lb = (k == ~0ull) ? CDTW_INF : 0.f;  // empty block: never started
    c.lbk = 0.f;                           // no cumulative bound for seeds
    cands[i] = c;
}

// Warp-aggregated append of the windows whose LB_Kim is below the best-so-far.
__global__ void __launch_bounds__(256)
compact_kim_kernel(const float* __restrict__ lbkim, int Nw, const unsigned long long* key,
                   int* __restrict__ q1, int* __restrict__ n1) {
    // a lane tests four consecutive windows (one 16-byte load; lbkim is
    // 256-byte aligned), a warp reserves its survivors with one atomic
    const float bsf = load_bsf(key);
    const int lane = threadIdx.x & 31;
    const int nvec = (Nw + 3) >> 2;
    const int stride = gridDim.x * blockDim.x;
    for (int base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31; base < nvec; base += stride) {
        const int v = base + lane;
        const int64_t w0 = 4 * (int64_t)v;
        float4 f = make_float4(INFINITY, INFINITY, INFINITY, INFINITY);
        if (w0 + 3 < Nw) {
            f = __ldg(reinterpret_cast<const float4*>(lbkim) + v);
        } else if (w0 < Nw) {
            f.x = lbkim[w0];
            if (w0 + 1 < Nw) f.y = lbkim[w0 + 1];
            if (w0 + 2 < Nw) f.z = lbkim[w0 + 2];
        }
        const unsigned k = (f.x * kLbSlack < bsf ? 1u : 0u) | (f.y * kLbSlack < bsf ? 2u : 0u) |
                           (f.z * kLbSlack < bsf ? 4u : 0u) | (f.w * kLbSlack < bsf ? 8u : 0u);
        const int c = __popc(k);
        int pre = c;  // inclusive prefix over the lanes
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, pre, o);
            if (lane >= o) pre += t;
        }
        const int tot = __shfl_sync(0xffffffffu, pre, 31);
        if (!tot) continue;
        int at = 0;
        if (lane == 31) at = atomicAdd(n1, tot);
        at = __shfl_sync(0xffffffffu, at, 31) + pre - c;
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (k & (1u << j)) q1[at++] = (int)w0 + j;
    }
}

// Forward + reverse LB_Keogh of the compacted windows; survivors -> q2.
template <bool EU>
__global__ void __launch_bounds__(256)
keogh_filter_kernel(const float* __restrict__ x, const double* __restrict__ mu,
                    const float* __restrict__ sigma, const float* __restrict__ zq,
                    const float2* __restrict__ qenv, const float2* __restrict__ xenv,
                    const float* __restrict__ lbkim, int M, const int* __restrict__ q1,
                    const int* __restrict__ n1p, const unsigned long long* key,
                    Cand* __restrict__ q2, int* __restrict__ n2, int sparse_max) {
    const int n1 = *(const volatile int*)n1p;
    if (n1 <= sparse_max) return;  // keogh_sparse_kernel takes few survivors
    const float bsf = load_bsf(key);
    const float lim = bsf / kLbSlack;  // bound value at which a window is pruned
    const int lane = threadIdx.x & 31;
    for (int base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31; base < n1;
         base += gridDim.x * blockDim.x) {
        const int i = base + lane;
        const bool valid = i < n1;
        const int w = valid ? q1[i] : q1[0];
        const Norm nm = make_norm(mu[w], sigma[w]);
        const float* __restrict__ xw = x + w;
        const float2* __restrict__ ew = xenv + w;
        float af = 0.f, ar = 0.f;
        auto term = [&](int k) {
            const float z = znorm(nm, __ldg(xw + k));
            const float2 e = __ldg(qenv + k);
            const float df = max3f(z - e.y, e.x - z, 0.f);
            af = EU ? fmaf(df, df, af) : af + df;
            const float2 d = __ldg(ew + k);
            const float q = __ldg(zq + k);
            const float dr = max3f(q - znorm(nm, d.y), znorm(nm, d.x) - q, 0.f);
            ar = EU ? fmaf(dr, dr, ar) : ar + dr;
        };
        int k0 = 0;
        // blocks of 16 samples, unrolled so their loads are all in flight
        // together; a warp-uniform early exit after each block
        for (; k0 + 16 <= M; k0 += 16) {
#pragma unroll
            for (int u = 0; u < 16; ++u) term(k0 + u);
            if (__all_sync(0xffffffffu, !valid || fmaxf(af, ar) >= lim)) break;
        }
        if (k0 + 16 > M && !__all_sync(0xffffffffu, !valid || fmaxf(af, ar) >= lim))
            for (int k = k0; k < M; ++k) term(k);
        const float lb = fmaxf(lbkim[w], fmaxf(af, ar));
        const bool keep = valid && lb < lim;
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (!m) continue;
        int at = 0;
        if (lane == 0) at = atomicAdd(n2, __popc(m));
        at = __shfl_sync(0xffffffffu, at, 0);
        if (keep) {
            Cand c;
            c.w = w;
            c.lb = lb;
            c.lbk = af;
            q2[at + __popc(m & ((1u << lane) - 1))] = c;
        }
    }
}

__device__ __forceinline__ float warp_sum_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

constexpr int kSparseMaxWarps = 16;  // warps per block of keogh_sparse_kernel (at most)

// Forward + reverse LB_Keogh for few LB_Kim survivors (at most sparse_max,
// scattered over the stream): a warp per window, lanes over the window's
// samples (coalesced).  The forward bound first, abandoned once its running
// sum passes the best-so-far; then, for the windows still below, the reverse
// bound against the +-W envelope of the window's own span of the stream,
// x[w-W, w+M-1+W] clipped to [0, N) (the values env_window_kernel computes
// for the whole stream), built in shared memory.  Survivors -> q2 as in
// keogh_filter_kernel.  Two ways to the envelope, the same values:
//  * VH (wide bands): van Herk / Gil-Werman blocks of 2W+1 positions, prefix
//    and suffix extrema per lane chunk (about five operations per position
//    at any W); 4 * S floats of shared memory per warp, S >= M + 2W.
//  * otherwise: log2(2W+1) doubling passes in place; 2 * S floats per warp,
//    so twice the warps per SM, which wins while the passes are few.
// Bounds are checked every 128 samples; a lane's loads for 256 are issued
// together.
template <bool EU, bool VH>
__global__ void __launch_bounds__(32 * kSparseMaxWarps, 1)
keogh_sparse_kernel(const float* __restrict__ x, int64_t N, const double* __restrict__ mu,
                    const float* __restrict__ sigma, const float* __restrict__ zq,
                    const float2* __restrict__ qenv, const float* __restrict__ lbkim, int M, int W,
                    int S, const int* __restrict__ q1, const int* __restrict__ n1p,
                    const unsigned long long* key, Cand* __restrict__ q2, int* __restrict__ n2,
                    int sparse_max) {
    extern __shared__ float ksm[];
    const int n1 = *(const volatile int*)n1p;
    if (n1 > sparse_max) return;  // keogh_filter_kernel takes many survivors
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    float* lo = ksm + (size_t)wib * (VH ? 4 : 2) * S;
    float* hi = lo + S;
    float* plo = hi + S;  // VH only
    float* phi = plo + S;
    const float lim = load_bsf(key) / kLbSlack;
    const int K = 2 * W + 1, span = M + 2 * W;
    int p = 1;  // doubling: the largest power of two <= K
    while (2 * p <= K) p *= 2;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int i = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < n1;
         i += nwarps) {
        const int w = q1[i];
        const Norm nm = make_norm(mu[w], sigma[w]);
        const float* __restrict__ xw = x + w;
        // forward LB_Keogh
        float af = 0.f, tf = 0.f;
        bool pruned = false;
        for (int k0 = 0; k0 < M && !pruned; k0 += 256) {
            float xv[8];
            float2 ev[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int k = min(k0 + 32 * u + lane, M - 1);
                xv[u] = __ldg(xw + k);
                ev[u] = __ldg(qenv + k);
            }
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                if (pruned || k0 + 128 * h >= M) break;  // warp-uniform
#pragma unroll
                for (int u = 4 * h; u < 4 * h + 4; ++u) {
                    if (k0 + 32 * u + lane < M) {
                        const float z = znorm(nm, xv[u]);
                        const float df = max3f(z - ev[u].y, ev[u].x - z, 0.f);
                        af = EU ? fmaf(df, df, af) : af + df;
                    }
                }
                tf = warp_sum_f(af);
                pruned = tf >= lim;
            }
        }
        if (pruned) continue;
        // the window's span of the stream (+inf / -inf outside the stream)
        for (int s0 = 0; s0 < span; s0 += 256) {
            float v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int64_t g = (int64_t)w - W + s0 + 32 * u + lane;
                v[u] = __ldg(x + min(max(g, (int64_t)0), N - 1));
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int e = s0 + 32 * u + lane;
                const int64_t g = (int64_t)w - W + e;
                const bool in = g >= 0 && g < N;
                if (e < span) {
                    lo[e] = in ? v[u] : CDTW_INF;
                    hi[e] = in ? v[u] : -CDTW_INF;
                }
            }
        }
        __syncwarp();
        if constexpr (VH) {
            // blocks of K consecutive span positions: extrema from each block
            // start (prefix, into plo / phi) and to each block end (suffix, in
            // place); the window [k, k+K) covers the end of one block and the
            // start of the next: env(k) = ext(suffix[k], prefix[k+K-1]).  A lane
            // scans a contiguous chunk of CH (odd: conflict-free) positions;
            // the open block's extremum crosses chunks by a segmented warp scan.
            const int CH = ((span + 31) / 32) | 1;
            const int e0 = min(lane * CH, span), e1 = min(e0 + CH, span);
            {  // prefix extrema within blocks, then the carry from earlier chunks
                float rl = CDTW_INF, rh = -CDTW_INF;
                int first = e1;  // first block start in the chunk
                int r = e0 % K;  // position in the block
    #pragma unroll 4
                for (int e = e0; e < e1; ++e) {
                    const bool s = r == 0;
                    const float vl = lo[e], vh = hi[e];
                    rl = fminf(s ? CDTW_INF : rl, vl);
                    rh = fmaxf(s ? -CDTW_INF : rh, vh);
                    if (s) first = min(first, e);
                    plo[e] = rl;
                    phi[e] = rh;
                    r = (r == K - 1) ? 0 : r + 1;
                }
                bool head = first < e1;  // the scan restarts at a chunk holding a block start
                float sl = rl, sh = rh;
    #pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const float tl = __shfl_up_sync(0xffffffffu, sl, o);
                    const float th = __shfl_up_sync(0xffffffffu, sh, o);
                    const bool tf = __shfl_up_sync(0xffffffffu, head, o);
                    if (lane >= o && !head) {
                        sl = fminf(sl, tl);
                        sh = fmaxf(sh, th);
                    }
                    if (lane >= o) head = head || tf;
                }
                float cl = __shfl_up_sync(0xffffffffu, sl, 1);
                float cr = __shfl_up_sync(0xffffffffu, sh, 1);
                if (lane == 0) {
                    cl = CDTW_INF;
                    cr = -CDTW_INF;
                }
                for (int e = e0; e < first; ++e) {
                    plo[e] = fminf(plo[e], cl);
                    phi[e] = fmaxf(phi[e], cr);
                }
            }
            {  // suffix extrema within blocks (in place), then the later chunks' carry
                float rl = CDTW_INF, rh = -CDTW_INF;
                int last = e0 - 1;  // last block end in the chunk
                int r = (e1 - 1) % K;
    #pragma unroll 4
                for (int e = e1 - 1; e >= e0; --e) {
                    const bool s = r == K - 1 || e == span - 1;
                    const float vl = lo[e], vh = hi[e];
                    rl = fminf(s ? CDTW_INF : rl, vl);
                    rh = fmaxf(s ? -CDTW_INF : rh, vh);
                    if (s) last = max(last, e);
                    lo[e] = rl;
                    hi[e] = rh;
                    r = (r == 0) ? K - 1 : r - 1;
                }
                bool head = last >= e0;
                float sl = rl, sh = rh;
    #pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const float tl = __shfl_down_sync(0xffffffffu, sl, o);
                    const float th = __shfl_down_sync(0xffffffffu, sh, o);
                    const bool tf = __shfl_down_sync(0xffffffffu, head, o);
                    if (lane + o < 32 && !head) {
                        sl = fminf(sl, tl);
                        sh = fmaxf(sh, th);
                    }
                    if (lane + o < 32) head = head || tf;
                }
                float cl = __shfl_down_sync(0xffffffffu, sl, 1);
                float cr = __shfl_down_sync(0xffffffffu, sh, 1);
                if (lane == 31) {
                    cl = CDTW_INF;
                    cr = -CDTW_INF;
                }
                for (int e = last + 1; e < e1; ++e) {
                    lo[e] = fminf(lo[e], cl);
                    hi[e] = fmaxf(hi[e], cr);
                }
            }
        } else {
            // min / max of 2^j positions from e, j = 1.. log2(p), in place
            // (chunks in increasing order: a partner e + q > e is never
            // rewritten before it is read)
            for (int q = 1; q < p; q *= 2) {
                for (int e0 = 0; e0 < span - q; e0 += 32) {
                    const int e = e0 + lane;
                    float a = 0.f, b = 0.f;
                    if (e < span - q) {
                        a = fminf(lo[e], lo[e + q]);
                        b = fmaxf(hi[e], hi[e + q]);
                    }
                    __syncwarp();
                    if (e < span - q) {
                        lo[e] = a;
                        hi[e] = b;
                    }
                    __syncwarp();
                }
            }
        }
        __syncwarp();
        // reverse LB_Keogh: the query against the window's envelope
        float ar = 0.f, tr = 0.f;
        for (int k0 = 0; k0 < M && !pruned; k0 += 256) {
            float qv[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) qv[u] = __ldg(zq + min(k0 + 32 * u + lane, M - 1));
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                if (pruned || k0 + 128 * h >= M) break;  // warp-uniform
#pragma unroll
                for (int u = 4 * h; u < 4 * h + 4; ++u) {
                    const int k = k0 + 32 * u + lane;
                    if (k < M) {
                        float L, U;
                        if constexpr (VH) {
                            L = fminf(lo[k], plo[k + K - 1]);
                            U = fmaxf(hi[k], phi[k + K - 1]);
                        } else {
                            L = fminf(lo[k], lo[k + K - p]);
                            U = fmaxf(hi[k], hi[k + K - p]);
                        }
                        const float dr =
                            max3f(qv[u] - znorm(nm, U), znorm(nm, L) - qv[u], 0.f);
                        ar = EU ? fmaf(dr, dr, ar) : ar + dr;
                    }
                }
                tr = warp_sum_f(ar);
                pruned = tr >= lim;
            }
        }
        __syncwarp();  // the span buffer is rewritten for the next window
        if (pruned) continue;
        const float lb = fmaxf(lbkim[w], fmaxf(tf, tr));
        if (lane == 0 && lb < lim) {
            Cand c;
            c.w = w;
            c.lb = lb;
            c.lbk = tf;
            q2[atomicAdd(n2, 1)] = c;
        }
    }
}

constexpr int kSparseSpanMax = 6144;  // M + 2W of the per-window envelope (96 KB a warp)
constexpr int kSparseVHMinBand = 301;  // 2W+1 from which the van Herk blocks serve it
// The dense regime (stream envelope + a thread per survivor) was also tried
// from a per-window work estimate (span x doubling passes): at M=1024, W=102
// and 204 it measured no faster than the per-window envelopes (586 against
// 548 us; 1.17 against 0.83 ms per search), so the choice stays by count.

// Forward + reverse LB_Keogh of the LB_Kim survivors q1 (count *n1, known
// only on the device) into q2 / *n2: up to sparse_max survivors a warp per
// window with the window's own envelope (keogh_sparse_kernel), above that the
// stream envelope of the whole stream and a thread per window
// (keogh_filter_kernel).  Both are launched; each returns at once outside its
// regime, as does the stream envelope below it.
int launch_keogh(cdtw_handle h, const float* x, int64_t N, const double* mu, const float* sigma,
                 bool euclid, const SearchWs& ws) {
    const QueryPack& q = h->q;
    const int M = q.M, W = q.W;
    const int span = M + 2 * W;
    const int S = (int)round_up(span, 4);
    const int sparse_max =
        span <= kSparseSpanMax ? (int)std::min<int64_t>(N / 256, (int64_t)1 << 18) : -1;
    CDTW_TRY(launch_stream_envelope(h, x, N, W, ws.envscratch, ws.xenv, ws.ctr + 0, sparse_max));
    const int grid = h->sm_count * 8;
    if (euclid)
        keogh_filter_kernel<true><<<grid, 256, 0, h->stream>>>(
            x, mu, sigma, q.zq, q.env, ws.xenv, ws.lbkim, M, ws.q1, ws.ctr + 0, ws.key, ws.q2,
            ws.ctr + 1, sparse_max);
    else
        keogh_filter_kernel<false><<<grid, 256, 0, h->stream>>>(
            x, mu, sigma, q.zq, q.env, ws.xenv, ws.lbkim, M, ws.q1, ws.ctr + 0, ws.key, ws.q2,
            ws.ctr + 1, sparse_max);
    CDTW_LAUNCH(h, "keogh_filter_kernel");
    if (sparse_max <= 0) return CDTW_OK;
    // van Herk blocks from kSparseVHMinBand (measured: the doubling passes
    // are faster at W <= 51 — 39 against 65 us at M=512 — and, with the
    // blocks sized below, at W = 102 — the M=1024 search 0.754 against
    // 0.787 ms, M=512 the same; van Herk is faster at W = 204)
    const bool vh = 2 * W + 1 >= kSparseVHMinBand;
    const int64_t per_warp = (int64_t)(vh ? 4 : 2) * S * sizeof(float);  // bytes
    auto k = vh ? (euclid ? keogh_sparse_kernel<true, true> : keogh_sparse_kernel<false, true>)
                : (euclid ? keogh_sparse_kernel<true, false> : keogh_sparse_kernel<false, false>);
    // warps per block for the most warps per SM: shared memory per SM and per
    // block (less the per-block reservation), registers, the warp limit
    int smem_sm = 0, smem_blk = 0, resv = 0, warps_sm = 0, blocks_sm = 0;
    CDTW_CUDA(h, cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor,
                                        h->device));
    CDTW_CUDA(h, cudaDeviceGetAttribute(&smem_blk, cudaDevAttrMaxSharedMemoryPerBlockOptin,
                                        h->device));
    CDTW_CUDA(h, cudaDeviceGetAttribute(&resv, cudaDevAttrReservedSharedMemoryPerBlock,
                                        h->device));
    CDTW_CUDA(h, cudaDeviceGetAttribute(&warps_sm, cudaDevAttrMaxThreadsPerMultiProcessor,
                                        h->device));
    CDTW_CUDA(h, cudaDeviceGetAttribute(&blocks_sm, cudaDevAttrMaxBlocksPerMultiprocessor,
                                        h->device));
    warps_sm /= 32;
    cudaFuncAttributes fa;
    CDTW_CUDA(h, cudaFuncGetAttributes(&fa, (const void*)k));
    const int64_t regs_warp = (int64_t)((fa.numRegs + 7) / 8 * 8) * 32;
    const int64_t reg_warps = regs_warp > 0 ? 65536 / regs_warp : warps_sm;
    int wpb = 1;
    int64_t best = 0;
    for (int c = 1; c <= kSparseMaxWarps; ++c) {
        if (c * per_warp > smem_blk) break;
        const int64_t nb = std::min<int64_t>(
            std::min<int64_t>(smem_sm / (c * per_warp + resv), blocks_sm),
            std::min<int64_t>(warps_sm, reg_warps) / c);
        if (nb * c >= best) {  // ties: the larger block
            best = nb * c;
            wpb = c;
        }
    }
    const size_t smem = (size_t)wpb * per_warp;
    CDTW_CUDA(h, cudaFuncSetAttribute((const void*)k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
    int per_sm = 0;
    CDTW_CUDA(h, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)k, 32 * wpb,
                                                               smem));
    const int64_t blocks = std::max<int64_t>(
        1, std::min<int64_t>(div_up(sparse_max, wpb), (int64_t)std::max(per_sm, 1) * h->sm_count));
    k<<<(unsigned)blocks, 32 * wpb, smem, h->stream>>>(x, N, mu, sigma, q.zq, q.env, ws.lbkim, M,
                                                       W, S, ws.q1, ws.ctr + 0, ws.key, ws.q2,
                                                       ws.ctr + 1, sparse_max);
    CDTW_LAUNCH(h, "keogh_sparse_kernel");
    return CDTW_OK;
}

// The survivors of the bounds run as pairwise wavefronts (at most
// kWaveSurvivors of them) when the band fits the pairwise forward and a
// window has at least kWaveMinCells band cells: a thread per window is then
// latency-bound.
bool wave_eligible(int M, int W) {
    const int Wp = std::min(W, M - 1);
    const double wcells = (double)M * (2.0 * Wp + 1.0) - (double)Wp * (Wp + 1.0);
    return Wp <= CDTW_PAIR_MAX_BAND && M <= CDTW_MAX_QUERY && wcells >= kWaveMinCells;
}

size_t carve_search(int64_t N, int64_t Nw, int M, int W, SearchWs* ws, char* base) {
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off = (size_t)round_up((int64_t)(off + bytes), 256);
        return base ? base + o : nullptr;
    };
    const int64_t nblk = div_up(Nw, kKimBlock);
    ws->lbkim = (float*)take(sizeof(float) * Nw);
    ws->seeds = (unsigned long long*)take(sizeof(unsigned long long) * nblk);
    ws->bmax = (unsigned*)take(sizeof(unsigned) * nblk);
    ws->seed_cands = (Cand*)take(sizeof(Cand) * nblk);
    ws->q1 = (int*)take(sizeof(int) * Nw);
    ws->q2 = (Cand*)take(sizeof(Cand) * Nw);
    ws->xenv = (float2*)take(sizeof(float2) * N);
    ws->envscratch = (float*)take(stream_envelope_scratch_bytes(N));
    ws->ctr = (int*)take(sizeof(int) * 8);
    ws->key = (unsigned long long*)take(2 * sizeof(unsigned long long));  // [1]: seeds
    // rows of the seed windows (at most one per LB_Kim block, kSeedMax) and,
    // when that pass can run for this (M, W), of the survivors run as
    // wavefronts (at most kWaveSurvivors)
    const int64_t rows = wave_eligible(M, W)
                             ? std::min<int64_t>(Nw, std::max<int64_t>(kSeedMax, kWaveSurvivors))
                             : std::min<int64_t>(nblk, kSeedMax);
    ws->seed_cap = std::min<int64_t>(rows * M, kSeedZMax);
    ws->seed_z = (float*)take(sizeof(float) * ws->seed_cap);
    ws->seed_d = (float*)take(sizeof(float) * std::max(kSeedMax, kWaveSurvivors));
    return off;
}

// ---- top-k non-overlapping matches ------------------------------------------

// One seed per segment s: the smallest-LB_Kim window start in [2Ms, 2Ms + M).
// Seeds of different segments start at least M + 1 apart, so they never
// overlap.  One warp per segment.
__global__ void topk_seed_kernel(const float* __restrict__ lbkim, int Nw, int M, int nseg,
                                 int32_t* __restrict__ sidx) {
    const int lane = threadIdx.x & 31;
    const int s = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (s >= nseg) return;
    const int lo = 2 * M * s, hi = min(lo + M, Nw);
    unsigned long long best = ~0ull;
    for (int w = lo + lane; w < hi; w += 32) best = min(best, pack_key(lbkim[w], (uint32_t)w));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = min(best, __shfl_xor_sync(0xffffffffu, best, o));
    if (lane == 0) sidx[s] = best == ~0ull ? lo : (int32_t)(uint32_t)best;
}

__global__ void cands_to_idx_kernel(const Cand* __restrict__ c, int n, int32_t* __restrict__ idx) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) idx[i] = c[i].w;
}

// Windows whose cDTW is at most T, as packed (distance, window) keys.
__global__ void collect_kernel(const float* __restrict__ d, const int32_t* __restrict__ idx,
                               int n, float T, unsigned long long* __restrict__ hits,
                               int* __restrict__ nh, int cap) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !(d[i] <= T)) return;
    const int at = atomicAdd(nh, 1);
    if (at < cap) hits[at] = pack_key(d[i], (uint32_t)idx[i]);
}

struct TopkWs {
    int32_t* sidx;
    float* sd;
    int32_t* idx;
    float* d;
    unsigned long long* hits;
    int* nh;
};

size_t carve_topk(int64_t N, int64_t Nw, int M, int W, int64_t cap, SearchWs* sw, TopkWs* tw,
                  char* base) {
    size_t off = carve_search(N, Nw, M, W, sw, base);
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off = (size_t)round_up((int64_t)(off + bytes), 256);
        return base ? base + o : nullptr;
    };
    const int64_t nseg = div_up(Nw, 2 * (int64_t)M);
    tw->sidx = (int32_t*)take(sizeof(int32_t) * nseg);
    tw->sd = (float*)take(sizeof(float) * nseg);
    tw->idx = (int32_t*)take(sizeof(int32_t) * Nw);
    tw->d = (float*)take(sizeof(float) * Nw);
    tw->hits = (unsigned long long*)take(sizeof(unsigned long long) * cap);
    tw->nh = (int*)take(sizeof(int) * 2);
    return off;
}

int64_t topk_cap(int64_t Nw) { return std::min<int64_t>(Nw, (int64_t)1 << 24); }

}  // namespace

size_t topk_workspace_bytes(int64_t N, int M, int W) {
    SearchWs sw;
    TopkWs tw;
    const int64_t Nw = N - M + 1;
    return carve_topk(N, Nw, M, W, topk_cap(Nw), &sw, &tw, nullptr);
}

// Greedy non-overlapping selection over the (distance, window) keys in
// ascending order: a window overlapping an accepted one is skipped, and the
// selection stops at k.  The keys are unique; only the prefix the greedy
// consumes is ordered: nth_element splits off the next smallest block, which
// is sorted and scanned, the block doubling until k windows are accepted.
static void greedy_picks(std::vector<unsigned long long>& hits, int k, int M,
                         std::vector<unsigned long long>* picks) {
    std::set<int64_t> taken;
    picks->clear();
    size_t lo = 0, block = std::max<size_t>(4096, (size_t)16 * (size_t)k);
    while (lo < hits.size() && (int)picks->size() < k) {
        const size_t hi = std::min(hits.size(), lo + block);
        if (hi < hits.size()) std::nth_element(hits.begin() + lo, hits.begin() + hi, hits.end());
        std::sort(hits.begin() + lo, hits.begin() + hi);
        for (size_t i = lo; i < hi && (int)picks->size() < k; ++i) {
            const unsigned long long key = hits[i];
            const int64_t w = (int64_t)(uint32_t)key;
            auto it = taken.lower_bound(w - M + 1);
            if (it != taken.end() && *it < w + M) continue;  // overlaps an accepted window
            taken.insert(w);
            picks->push_back(key);
        }
        lo = hi;
        block *= 2;
    }
}

// Top-k non-overlapping matches of the handle's query.  Greedy selection in
// (distance, window) order with windows overlapping an accepted one skipped.
// The candidate threshold T is the 2k-th smallest cDTW among the segment
// seeds: they are pairwise non-overlapping, and each accepted match overlaps
// at most two of them, so every one of the first k greedy picks has a
// distance <= T and all windows above T can be pruned.  Host-synchronous.
int run_topk(cdtw_handle h, const float* x, int64_t N, const double* mu, const float* sigma,
             bool euclid, int k, char* ws_base, std::vector<unsigned long long>* picks) {
    const QueryPack& q = h->q;
    const int M = q.M;
    const int64_t Nw = N - M + 1;
    SearchWs ws;
    TopkWs tw;
    const int64_t cap = topk_cap(Nw);
    carve_topk(N, Nw, M, q.W, cap, &ws, &tw, ws_base);
    const int nseg = (int)div_up(Nw, 2 * (int64_t)M);
    // 1. LB_Kim of every window, seeds per segment, their exact cDTW
    CDTW_TRY(launch_lb_kim(h, x, N, mu, sigma, nullptr, Nw, euclid, ws.lbkim, ws.seeds,
                           ws.bmax));
    topk_seed_kernel<<<(unsigned)div_up((int64_t)nseg * 32, 256), 256, 0, h->stream>>>(
        ws.lbkim, (int)Nw, M, nseg, tw.sidx);
    CDTW_LAUNCH(h, "topk_seed_kernel");
    CDTW_TRY(launch_cdtw_windows(h, x, N, mu, sigma, tw.sidx, nseg, euclid, tw.sd));
    std::vector<float> sd(nseg);
    CDTW_CUDA(h, cudaMemcpyAsync(sd.data(), tw.sd, sizeof(float) * nseg, cudaMemcpyDeviceToHost,
                                 h->stream));
    CDTW_CUDA(h, cudaStreamSynchronize(h->stream));
    float T = INFINITY;
    if ((int64_t)nseg >= 2 * (int64_t)k) {
        std::nth_element(sd.begin(), sd.begin() + (2 * k - 1), sd.end());
        T = sd[2 * k - 1];
    }
    // 2. bounds against T (the key holds T as the best-so-far)
    const unsigned long long tkey = pack_key(T, 0xffffffffu);
    CDTW_CUDA(h, cudaMemsetAsync(ws.ctr, 0, sizeof(int) * 8, h->stream));
    CDTW_CUDA(h, cudaMemsetAsync(tw.nh, 0, sizeof(int) * 2, h->stream));
    CDTW_CUDA(h, cudaMemcpyAsync(ws.key, &tkey, sizeof(tkey), cudaMemcpyHostToDevice, h->stream));
    const int grid = h->sm_count * 8;
    compact_kim_kernel<<<grid, 256, 0, h->stream>>>(ws.lbkim, (int)Nw, ws.key, ws.q1, ws.ctr + 0);
    CDTW_LAUNCH(h, "compact_kim_kernel");
    CDTW_TRY(launch_keogh(h, x, N, mu, sigma, euclid, ws));
    int cnt[2];
    CDTW_CUDA(h, cudaMemcpyAsync(cnt, ws.ctr, sizeof(cnt), cudaMemcpyDeviceToHost, h->stream));
    CDTW_CUDA(h, cudaStreamSynchronize(h->stream));
    h->last_counts[0] = Nw;
    h->last_counts[1] = cnt[0];
    h->last_counts[2] = cnt[1];
    // 3. exact cDTW of the survivors, those <= T collected
    const int ns = cnt[1];
    if (ns > 0) {
        cands_to_idx_kernel<<<(unsigned)div_up(ns, 256), 256, 0, h->stream>>>(ws.q2, ns, tw.idx);
        CDTW_LAUNCH(h, "cands_to_idx_kernel");
        CDTW_TRY(launch_cdtw_windows(h, x, N, mu, sigma, tw.idx, ns, euclid, tw.d));
        collect_kernel<<<(unsigned)div_up(ns, 256), 256, 0, h->stream>>>(tw.d, tw.idx, ns, T,
                                                                        tw.hits, tw.nh, (int)cap);
        CDTW_LAUNCH(h, "collect_kernel");
    }
    int nh = 0;
    CDTW_CUDA(h, cudaMemcpyAsync(&nh, tw.nh, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CDTW_CUDA(h, cudaStreamSynchronize(h->stream));
    if (nh > cap)
        return set_error(h, CDTW_EUNSUPPORTED, "%d windows under the top-k threshold (limit %lld)",
                         nh, (long long)cap);
    std::vector<unsigned long long> hits(nh);
    if (nh > 0) {
        CDTW_CUDA(h, cudaMemcpyAsync(hits.data(), tw.hits, sizeof(unsigned long long) * nh,
                                     cudaMemcpyDeviceToHost, h->stream));
        CDTW_CUDA(h, cudaStreamSynchronize(h->stream));
    }
    // 4. greedy non-overlapping selection, lowest (distance, window) first
    greedy_picks(hits, k, M, picks);
    return CDTW_OK;
}

// Workspace of run_topk_device: that of run_topk plus the re-scored previous
// picks, the threshold and the accepted-window buckets of the greedy.
namespace {
struct TopkDevWs {
    float* prev_d;
    float* T;
    int* acc;
    int nbuckets;
};
size_t carve_topk_device(int64_t N, int M, int W, int k2, SearchWs* sw, TopkWs* tw,
                         TopkDevWs* dw, char* base) {
    const int64_t Nw = N - M + 1;
    size_t off = carve_topk(N, Nw, M, W, topk_cap(Nw), sw, tw, base);
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off = (size_t)round_up((int64_t)(off + bytes), 256);
        return base ? base + o : nullptr;
    };
    dw->prev_d = (float*)take(sizeof(float) * std::max(k2, 1));
    dw->T = (float*)take(sizeof(float));
    dw->nbuckets = (int)div_up(Nw, M);
    dw->acc = (int*)take(sizeof(int) * ((size_t)dw->nbuckets + 2));
    return off;
}
}  // namespace

size_t topk_device_workspace_bytes(int64_t N, int M, int W, int k2) {
    SearchWs sw;
    TopkWs tw;
    TopkDevWs dw;
    return carve_topk_device(N, M, W, k2, &sw, &tw, &dw, nullptr);
}

// The top-k search of run_topk with every step on the device (no host
// synchronisation, so it can be captured in a CUDA graph): the threshold T
// is selected on the device (and lowered to the largest re-scored distance
// of `prev`, a previous set of k2 non-overlapping windows, when *prev_n ==
// k2), the windows at distance <= T are collected by the early-abandoning
// search kernels into a hit list, and the greedy selection runs in one block
// (topk_device.cu).  The greedy continues to k2 picks over the same
// candidates: the first k (T from 2k of the seeds or of `prev`) are the exact
// greedy picks; all of them are non-overlapping, which is all the next call's
// threshold needs.  prev may alias picks and prev_n npicks.  *status: 0, or
// 1 when more windows than the hit list holds fell under T.
int run_topk_device(cdtw_handle h, const float* x, int64_t N, const double* mu,
                    const float* sigma, bool euclid, int k, int k2, char* ws_base,
                    const int32_t* prev, const int* prev_n, int32_t* picks, float* pick_d,
                    int* npicks, int* status) {
    const QueryPack& q = h->q;
    const int M = q.M;
    const int64_t Nw = N - M + 1;
    if (k < 1 || k2 < k || (prev && k2 < 2 * k))
        return set_error(h, CDTW_EINVAL, "device top-k: k=%d, k2=%d", k, k2);
    SearchWs ws;
    TopkWs tw;
    TopkDevWs dw;
    carve_topk_device(N, M, q.W, k2, &ws, &tw, &dw, ws_base);
    const int64_t cap = topk_cap(Nw);
    const int nseg = (int)div_up(Nw, 2 * (int64_t)M);
    CDTW_CUDA(h, cudaMemsetAsync(ws.ctr, 0, sizeof(int) * 8, h->stream));
    CDTW_CUDA(h, cudaMemsetAsync(tw.nh, 0, sizeof(int) * 2, h->stream));
    // 1. LB_Kim of every window, one seed per segment, their exact cDTW
    CDTW_TRY(launch_lb_kim(h, x, N, mu, sigma, nullptr, Nw, euclid, ws.lbkim));
    topk_seed_kernel<<<(unsigned)div_up((int64_t)nseg * 32, 256), 256, 0, h->stream>>>(
        ws.lbkim, (int)Nw, M, nseg, tw.sidx);
    CDTW_LAUNCH(h, "topk_seed_kernel");
    CDTW_TRY(launch_cdtw_windows(h, x, N, mu, sigma, tw.sidx, nseg, euclid, tw.sd));
    // 2. the threshold (the previous windows re-scored with this query)
    if (prev && prev_n)
        CDTW_TRY(launch_cdtw_windows(h, x, N, mu, sigma, prev, k2, euclid, dw.prev_d));
    CDTW_TRY(launch_topk_threshold(h, tw.sd, nseg, dw.prev_d, prev ? prev_n : nullptr, 2 * k,
                                   ws.key, dw.T));
    // 3. bounds against T, the survivors' cDTW collected as hits
    const int grid = h->sm_count * 8;
    compact_kim_kernel<<<grid, 256, 0, h->stream>>>(ws.lbkim, (int)Nw, ws.key, ws.q1, ws.ctr + 0);
    CDTW_LAUNCH(h, "compact_kim_kernel");
    CDTW_TRY(launch_keogh(h, x, N, mu, sigma, euclid, ws));
    HitSink sink;
    sink.hits = tw.hits;
    sink.n = tw.nh;
    sink.cap = (int)cap;
    CDTW_TRY(launch_cdtw_search(h, x, N, mu, sigma, ws.q2, ws.ctr + 1, ws.ctr + 3, (int)Nw,
                                euclid, ws.key, sink));
    // 4. greedy selection
    CDTW_CUDA(h, cudaMemsetAsync(dw.acc, 0xff, sizeof(int) * ((size_t)dw.nbuckets + 2),
                                 h->stream));
    return launch_topk_greedy(h, tw.hits, tw.nh, (int)cap, k2, M, dw.acc, picks, pick_d, npicks,
                              status);
}

size_t search_workspace_bytes(int64_t N, int M, int W) {
    SearchWs ws;
    return carve_search(N, N - M + 1, M, W, &ws, nullptr);
}

// Runs the whole pruned search; the result key and the stage counts stay on
// the device (ws key / counters) for the caller to read.
int run_search(cdtw_handle h, const float* x, int64_t N, const double* mu, const float* sigma,
               bool euclid, char* ws_base, unsigned long long** key_out, int** ctr_out,
               const unsigned long long* init_key) {
    const QueryPack& q = h->q;
    const int64_t Nw = N - q.M + 1;
    SearchWs ws;
    carve_search(N, Nw, q.M, q.W, &ws, ws_base);
    CDTW_CUDA(h, cudaMemsetAsync(ws.ctr, 0, sizeof(int) * 8, h->stream));
    CDTW_CUDA(h, cudaMemsetAsync(ws.key, 0xff, 2 * sizeof(unsigned long long), h->stream));
    if (init_key)
        CDTW_CUDA(h, cudaMemcpyAsync(ws.key, init_key, sizeof(unsigned long long),
                                     cudaMemcpyDeviceToDevice, h->stream));
    // 1. LB_Kim of every window + per-block seeds
    const int64_t nblk = div_up(Nw, kKimBlock);
    CDTW_TRY(launch_lb_kim_all(h, x, N, mu, sigma, euclid, ws.lbkim, ws.seeds, ws.bmax));
    // 2. cDTW of the seeds
    const int G = (int)std::max<int64_t>(1, div_up(nblk, seed_target(q.M, q.W)));
    const int nseed = (int)div_up(nblk, G);
    seeds_to_cands_kernel<<<(unsigned)div_up((int64_t)nseed * 32, 256), 256, 0, h->stream>>>(
        ws.seeds, ws.bmax, (int)nblk, G, ws.seed_cands, ws.ctr + 4, (unsigned*)ws.ctr + 5);
    CDTW_LAUNCH(h, "seeds_to_cands_kernel");
    // the seeds only bound the search from above (raised a little, with no
    // window): with few windows in flight their cDTW is latency-bound, so it
    // runs as pairwise wavefronts (a lane group per seed) when the band and
    // the seed windows fit, else on the search kernels (into a key of their
    // own, raised the same way).  The lane-group search kernel was measured
    // slower here than the wavefronts (M=512, W=51: 1.04 against 0.66 ms per
    // search).
    const int Wp = std::min(q.W, q.M - 1);
    if (Wp <= CDTW_PAIR_MAX_BAND && q.M <= CDTW_MAX_QUERY && nseed <= kSeedMax &&
        (int64_t)nseed * q.M <= ws.seed_cap) {
        seed_gather_kernel<<<(unsigned)div_up((int64_t)nseed * 32, 256), 256, 0, h->stream>>>(
            x, mu, sigma, ws.seed_cands, nseed, q.M, ws.seed_z);
        CDTW_LAUNCH(h, "seed_gather_kernel");
        CDTW_TRY(launch_pair_fwd(h, q.zq, ws.seed_z, nseed, q.M, Wp, euclid, ws.seed_d, nullptr,
                                 nullptr, nullptr, /*qstride=*/0));
        seed_bound_kernel<<<(unsigned)div_up(nseed, 256), 256, 0, h->stream>>>(
            ws.seed_d, ws.seed_cands, nseed, q.M, ws.key);
        CDTW_LAUNCH(h, "seed_bound_kernel");
    } else {
        CDTW_TRY(launch_cdtw_search(h, x, N, mu, sigma, ws.seed_cands, ws.ctr + 4, ws.ctr + 2,
                                    nseed, euclid, ws.key + 1));
        seed_key_bound_kernel<<<1, 1, 0, h->stream>>>(ws.key + 1, q.M, ws.key);
        CDTW_LAUNCH(h, "seed_key_bound_kernel");
    }
    // 3. compaction by LB_Kim
    const int grid = h->sm_count * 8;
    compact_kim_kernel<<<grid, 256, 0, h->stream>>>(ws.lbkim, (int)Nw, ws.key, ws.q1, ws.ctr + 0);
    CDTW_LAUNCH(h, "compact_kim_kernel");
    // 4. LB_Keogh forward + reverse
    CDTW_TRY(launch_keogh(h, x, N, mu, sigma, euclid, ws));
    // 5. cDTW of the survivors: as pairwise wavefronts when at most `wcap`
    //    remain and a window is long enough that a thread per window is
    //    latency-bound, else with early abandoning
    //    When the band runs on the lane-group search kernel (which abandons
    //    windows early, group by group), only a handful of survivors go to
    //    the wavefronts: measured at M=1024, W=204, the wavefronts of 4373
    //    survivors took 0.53 ms.
    int wcap = (int)std::min<int64_t>(kWaveSurvivors, ws.seed_cap / q.M);
    if (choose_variant(h, q.W) == CDTW_VARIANT_LANE) wcap = std::min(wcap, kWaveFew);
    if (wave_eligible(q.M, q.W) && wcap >= 32) {
        wave_gather_kernel<<<(unsigned)div_up((int64_t)wcap * 32, 256), 256, 0, h->stream>>>(
            x, mu, sigma, ws.q2, ws.ctr + 1, wcap, q.M, ws.seed_z, ws.ctr + 3);
        CDTW_LAUNCH(h, "wave_gather_kernel");
        // a handful of survivors: the widest lane groups (shortest step);
        // more: the throughput shape (each launch gated to its range)
        const int few = std::min(wcap, kWaveFew);
        CDTW_TRY(launch_pair_fwd(h, q.zq, ws.seed_z, few, q.M, Wp, euclid, ws.seed_d, nullptr,
                                 nullptr, nullptr, /*qstride=*/0, ws.ctr + 1, few, -1,
                                 /*wide=*/true));
        if (wcap > few)
            CDTW_TRY(launch_pair_fwd(h, q.zq, ws.seed_z, wcap, q.M, Wp, euclid, ws.seed_d,
                                     nullptr, nullptr, nullptr, /*qstride=*/0, ws.ctr + 1, wcap,
                                     few));
        wave_keys_kernel<<<(unsigned)div_up(wcap, 256), 256, 0, h->stream>>>(
            ws.seed_d, ws.q2, ws.ctr + 1, wcap, ws.key);
        CDTW_LAUNCH(h, "wave_keys_kernel");
    }
    CDTW_TRY(launch_cdtw_search(h, x, N, mu, sigma, ws.q2, ws.ctr + 1, ws.ctr + 3, (int)Nw,
                                euclid, ws.key));
    if (key_out) *key_out = ws.key;
    if (ctr_out) *ctr_out = ws.ctr;
    return CDTW_OK;
}

}  // namespace cdtw
