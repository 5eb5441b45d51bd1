// Strip kernels (one window per thread, R-row strips, L2-resident rings):
// launchers for all listed windows and for the single-query search.  The
// device code and its description are in cdtw_strip.cuh.
#include "cdtw_strip.cuh"

namespace cdtw {

namespace {

__device__ __forceinline__ float* lane_ring(const StripArgs& a) {
    const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    return a.ring + (size_t)gwarp * a.P * 32 + (threadIdx.x & 31);
}

// All listed (or all) windows; persistent warps over chunks of 32 windows.
template <int R, bool EU>
__global__ void __launch_bounds__(kStripWarps * 32)
cdtw_strip_kernel(const StripArgs a) {
    float* ring = lane_ring(a);
    const int lane = threadIdx.x & 31;
    const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int chunk = gwarp; chunk * 32 < a.L; chunk += nwarps) {
        const int t_id = chunk * 32 + lane;
        if (t_id >= a.L) continue;  // lanes are independent in this mode
        const int w = a.idx ? a.idx[t_id] : t_id;
        if (w < 0 || w >= a.Nw) {  // a listed window outside the subject: NaN, no access
            a.out[t_id] = __int_as_float(0x7fc00000);
            continue;
        }
        bool alive = true;
        a.out[t_id] = strip_dtw<R, EU, false>(a, w, ring, nullptr, 0.f, alive, nullptr);
    }
}

// Search variant: persistent warps over a candidate list (see the register
// kernel's search variant for the protocol).
template <int R, bool EU>
__global__ void __launch_bounds__(kStripWarps * 32)
cdtw_strip_search_kernel(const StripArgs a, const float2* __restrict__ qenv,
                         const Cand* __restrict__ cands, const int* __restrict__ count,
                         int* __restrict__ work, unsigned long long* __restrict__ key,
                         const HitSink sink) {
    float* ring = lane_ring(a);
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
        const float res = strip_dtw<R, EU, true>(a, c.w, ring, qenv, c.lbk, alive, key);
        if (i < n && res < CDTW_INF) report_window(key, sink, res, (uint32_t)c.w);
    }
}

// Fill the common arguments; size the persistent grid and the ring slices.
template <class K>
int prepare_strip(cdtw_handle h, K k, const float* x, int64_t N, const double* mu,
                  const float* sigma, int R, int64_t work_items, StripArgs* a, int* blocks) {
    const QueryPack& q = h->q;
    a->x = x;
    a->mu = mu;
    a->sigma = sigma;
    a->qrev4 = (const float4*)q.qrev;
    a->qrev0 = q.qrev;
    a->lqr4 = q.lqr / 4;
    a->qbase = q.qrev_base;
    a->M = q.M;
    a->W = q.W;
    a->P = (int)round_up(2 * q.W + 2, R);
    a->Nw = (int)(N - q.M + 1);
    int per_sm = 0;
    CDTW_CUDA(h, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)k,
                                                               kStripWarps * 32, 0));
    const int64_t want = div_up(std::max<int64_t>(work_items, 1), kStripWarps * 32);
    *blocks = (int)std::max<int64_t>(
        1, std::min<int64_t>(want, (int64_t)std::max(per_sm, 1) * h->sm_count));
    const size_t ring_bytes = (size_t)(*blocks) * kStripWarps * a->P * 32 * sizeof(float);
    if (ring_bytes > h->ring_bytes) {
        CDTW_TRY(check_memory_limit(h, h->ring_bytes, ring_bytes, "strip rings"));
        if (h->ring) {
            CDTW_CUDA(h, cudaStreamSynchronize(h->stream));
            CDTW_CUDA(h, cudaFree(h->ring));
            h->ring = nullptr;
            h->ring_bytes = 0;
        }
        CDTW_CUDA(h, cudaMalloc(&h->ring, ring_bytes));
        h->ring_bytes = ring_bytes;
    }
    a->ring = (float*)h->ring;
    return CDTW_OK;
}

}  // namespace

int strip_rows_default(int W) { return W >= 63 ? 32 : 16; }

// Strip kernel launch for bands W >= R-1.  R in {16, 32}.
int launch_cdtw_strip(cdtw_handle h, const float* x, int64_t N, const double* mu,
                      const float* sigma, const int32_t* idx, int64_t L, bool euclid, int R,
                      float* out) {
    const QueryPack& q = h->q;
    if (R != 16 && R != 32) return set_error(h, CDTW_EINVAL, "strip rows must be 16 or 32");
    if (q.W < R - 1)
        return set_error(h, CDTW_EUNSUPPORTED, "strip kernel needs W >= R-1 (W=%d R=%d)", q.W, R);
    if (L <= 0) return CDTW_OK;
    using SK = void (*)(const StripArgs);
    SK k;
    if (R == 16) k = euclid ? cdtw_strip_kernel<16, true> : cdtw_strip_kernel<16, false>;
    else k = euclid ? cdtw_strip_kernel<32, true> : cdtw_strip_kernel<32, false>;
    StripArgs a;
    int blocks = 0;
    CDTW_TRY(prepare_strip(h, k, x, N, mu, sigma, R, L, &a, &blocks));
    a.idx = idx;
    a.L = (int)L;
    a.out = out;
    k<<<blocks, kStripWarps * 32, 0, h->stream>>>(a);
    CDTW_LAUNCH(h, "cdtw_strip_kernel");
    return CDTW_OK;
}

int launch_cdtw_strip_search(cdtw_handle h, const float* x, int64_t N, const double* mu,
                             const float* sigma, const Cand* cands, const int* count, int* work,
                             int max_count, bool euclid, int R, unsigned long long* key,
                             const HitSink& sink) {
    const QueryPack& q = h->q;
    if (R != 16 && R != 32) return set_error(h, CDTW_EINVAL, "strip rows must be 16 or 32");
    if (q.W < R - 1)
        return set_error(h, CDTW_EUNSUPPORTED, "strip kernel needs W >= R-1 (W=%d R=%d)", q.W, R);
    if (max_count <= 0) return CDTW_OK;
    using SK = void (*)(const StripArgs, const float2*, const Cand*, const int*, int*,
                        unsigned long long*, const HitSink);
    SK k;
    if (R == 16)
        k = euclid ? cdtw_strip_search_kernel<16, true> : cdtw_strip_search_kernel<16, false>;
    else
        k = euclid ? cdtw_strip_search_kernel<32, true> : cdtw_strip_search_kernel<32, false>;
    StripArgs a;
    int blocks = 0;
    CDTW_TRY(prepare_strip(h, k, x, N, mu, sigma, R, max_count, &a, &blocks));
    a.idx = nullptr;
    a.L = 0;
    a.out = nullptr;
    k<<<blocks, kStripWarps * 32, 0, h->stream>>>(a, q.env, cands, count, work, key, sink);
    CDTW_LAUNCH(h, "cdtw_strip_search_kernel");
    return CDTW_OK;
}

}  // namespace cdtw
