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
//   4. Forward LB_Keogh (query envelope) and reverse LB_Keogh (stream
//      envelope, as UCR_DTW_BIN.cpp:262-282) of those, with a warp-level exit
//      once every lane's bound passed the best-so-far; survivors keep their
//      best bound and their forward LB_Keogh.
//   5. cDTW of the survivors with early abandoning against the live
//      best-so-far, folded into the key.
// No sort, no host loop; graph-capturable launch sequence.
#include "common.cuh"

#include <algorithm>

namespace cdtw {

namespace {

struct SearchWs {
    float* lbkim = nullptr;
    unsigned long long* seeds = nullptr;
    Cand* seed_cands = nullptr;
    int* q1 = nullptr;
    Cand* q2 = nullptr;
    float2* xenv = nullptr;
    float* envscratch = nullptr;
    int* ctr = nullptr;  // [0] n1, [1] n2, [2] work seeds, [3] work main, [4] n seeds
    unsigned long long* key = nullptr;
};

constexpr int kKimBlock = 256;

// Seed candidates: the smallest LB_Kim window of each group of G blocks.
__global__ void seeds_to_cands_kernel(const unsigned long long* __restrict__ seeds, int nblk,
                                      int G, Cand* __restrict__ cands, int* __restrict__ nseeds) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = (nblk + G - 1) / G;
    if (i == 0) *nseeds = n;
    if (i >= n) return;
    unsigned long long k = ~0ull;
    for (int b = i * G; b < min(nblk, (i + 1) * G); ++b) k = min(k, seeds[b]);
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
    const float bsf = load_bsf(key);
    const int lane = threadIdx.x & 31;
    for (int base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31; base < Nw;
         base += gridDim.x * blockDim.x) {
        const int w = base + lane;
        const bool keep = w < Nw && lbkim[w] * kLbSlack < bsf;
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (!m) continue;
        int at = 0;
        if (lane == 0) at = atomicAdd(n1, __popc(m));
        at = __shfl_sync(0xffffffffu, at, 0);
        if (keep) q1[at + __popc(m & ((1u << lane) - 1))] = w;
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
                    Cand* __restrict__ q2, int* __restrict__ n2) {
    const int n1 = *(const volatile int*)n1p;
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
        for (int k0 = 0; k0 < M; k0 += 16) {
            const int k1 = min(k0 + 16, M);
            for (int k = k0; k < k1; ++k) {
                const float z = znorm(nm, __ldg(xw + k));
                const float2 e = __ldg(qenv + k);
                const float df = max3f(z - e.y, e.x - z, 0.f);
                af = EU ? fmaf(df, df, af) : af + df;
                const float2 d = __ldg(ew + k);
                const float q = __ldg(zq + k);
                const float dr = max3f(q - znorm(nm, d.y), znorm(nm, d.x) - q, 0.f);
                ar = EU ? fmaf(dr, dr, ar) : ar + dr;
            }
            if (__all_sync(0xffffffffu, !valid || fmaxf(af, ar) >= lim)) break;
        }
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

size_t carve_search(int64_t N, int64_t Nw, SearchWs* ws, char* base) {
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off = (size_t)round_up((int64_t)(off + bytes), 256);
        return base ? base + o : nullptr;
    };
    const int64_t nblk = div_up(Nw, kKimBlock);
    ws->lbkim = (float*)take(sizeof(float) * Nw);
    ws->seeds = (unsigned long long*)take(sizeof(unsigned long long) * nblk);
    ws->seed_cands = (Cand*)take(sizeof(Cand) * nblk);
    ws->q1 = (int*)take(sizeof(int) * Nw);
    ws->q2 = (Cand*)take(sizeof(Cand) * Nw);
    ws->xenv = (float2*)take(sizeof(float2) * N);
    ws->envscratch = (float*)take(stream_envelope_scratch_bytes(N));
    ws->ctr = (int*)take(sizeof(int) * 8);
    ws->key = (unsigned long long*)take(sizeof(unsigned long long));
    return off;
}

}  // namespace

size_t search_workspace_bytes(int64_t N, int M) {
    SearchWs ws;
    return carve_search(N, N - M + 1, &ws, nullptr);
}

// Runs the whole pruned search; the result key and the stage counts stay on
// the device (ws key / counters) for the caller to read.
int run_search(cdtw_handle h, const float* x, int64_t N, const double* mu, const float* sigma,
               bool euclid, char* ws_base, unsigned long long** key_out, int** ctr_out) {
    const QueryPack& q = h->q;
    const int64_t Nw = N - q.M + 1;
    SearchWs ws;
    carve_search(N, Nw, &ws, ws_base);
    CDTW_CUDA(h, cudaMemsetAsync(ws.ctr, 0, sizeof(int) * 8, h->stream));
    CDTW_CUDA(h, cudaMemsetAsync(ws.key, 0xff, sizeof(unsigned long long), h->stream));
    // 1. LB_Kim of every window + per-block seeds
    const int64_t nblk = div_up(Nw, kKimBlock);
    CDTW_TRY(launch_lb_kim(h, x, N, mu, sigma, nullptr, Nw, euclid, ws.lbkim, ws.seeds));
    // 2. cDTW of the seeds
    const int G = (int)std::max<int64_t>(1, div_up(nblk, seed_target(q.M, q.W)));
    const int nseed = (int)div_up(nblk, G);
    seeds_to_cands_kernel<<<(unsigned)div_up(nseed, 256), 256, 0, h->stream>>>(
        ws.seeds, (int)nblk, G, ws.seed_cands, ws.ctr + 4);
    CDTW_LAUNCH(h, "seeds_to_cands_kernel");
    CDTW_TRY(launch_cdtw_search(h, x, N, mu, sigma, ws.seed_cands, ws.ctr + 4, ws.ctr + 2,
                                nseed, euclid, ws.key));
    // 3. compaction by LB_Kim
    const int grid = h->sm_count * 8;
    compact_kim_kernel<<<grid, 256, 0, h->stream>>>(ws.lbkim, (int)Nw, ws.key, ws.q1, ws.ctr + 0);
    CDTW_LAUNCH(h, "compact_kim_kernel");
    // 4. LB_Keogh forward + reverse
    CDTW_TRY(launch_stream_envelope(h, x, N, q.W, ws.envscratch, ws.xenv));
    if (euclid)
        keogh_filter_kernel<true><<<grid, 256, 0, h->stream>>>(
            x, mu, sigma, q.zq, q.env, ws.xenv, ws.lbkim, q.M, ws.q1, ws.ctr + 0, ws.key, ws.q2,
            ws.ctr + 1);
    else
        keogh_filter_kernel<false><<<grid, 256, 0, h->stream>>>(
            x, mu, sigma, q.zq, q.env, ws.xenv, ws.lbkim, q.M, ws.q1, ws.ctr + 0, ws.key, ws.q2,
            ws.ctr + 1);
    CDTW_LAUNCH(h, "keogh_filter_kernel");
    // 5. cDTW of the survivors with early abandoning
    CDTW_TRY(launch_cdtw_search(h, x, N, mu, sigma, ws.q2, ws.ctr + 1, ws.ctr + 3, (int)Nw,
                                euclid, ws.key));
    if (key_out) *key_out = ws.key;
    if (ctr_out) *ctr_out = ws.ctr;
    return CDTW_OK;
}

}  // namespace cdtw
