// Device-side pieces of the top-k non-overlapping match search, so that the
// whole search runs without a host round trip (and can be captured in a
// CUDA graph): the candidate threshold by radix selection, and the greedy
// non-overlapping selection over the collected (distance, window) keys.
//
// Greedy selection: keys in ascending order; a window is accepted unless it
// overlaps (starts within M samples of) an accepted one; stop at k picks.
// Accepted windows are at least M apart, so with buckets of M consecutive
// window starts each bucket holds at most one of them, and a window w can
// only overlap accepted windows in the buckets w/M - 1, w/M and w/M + 1:
// the overlap test is three loads.  The keys are ordered only as far as the
// greedy consumes them: one block repeatedly radix-selects the next B
// smallest keys, sorts them in shared memory, tests them against the
// accepted windows in parallel and resolves the few that remain in key order
// with one warp (ballots over 32 keys at a time).
#include "common.cuh"

namespace cdtw {

namespace {

constexpr int kSelThreads = 1024;
constexpr int kGreedyB = 4096;  // keys ordered per round (32 KB of shared memory)

// Index (in an ascending order of n values) of the bucket that holds rank r:
// on return, *r is the rank inside that bucket.  hist: 256 counts.  Thread 0.
__device__ int pick_digit(const int* hist, int* r) {
    int cum = 0;
    for (int d = 0; d < 256; ++d) {
        if (cum + hist[d] > *r) {
            *r -= cum;
            return d;
        }
        cum += hist[d];
    }
    return 255;
}

// The (r+1)-th smallest of n non-negative floats (their bits order as
// unsigned ints), by four 8-bit radix passes.  All threads of the block get
// the result.
__device__ float select_rank_f32(const float* __restrict__ v, int n, int r, int* hist,
                                 unsigned* shared_prefix) {
    unsigned prefix = 0, mask = 0;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int d = threadIdx.x; d < 256; d += blockDim.x) hist[d] = 0;
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const unsigned u = __float_as_uint(v[i]);
            if ((u & mask) == prefix) atomicAdd(&hist[(u >> shift) & 255u], 1);
        }
        __syncthreads();
        if (threadIdx.x == 0) *shared_prefix = prefix | ((unsigned)pick_digit(hist, &r) << shift);
        __syncthreads();
        prefix = *shared_prefix;
        mask |= 255u << shift;  // (only thread 0's copy of r is used)
        __syncthreads();
    }
    return __uint_as_float(prefix);
}

// T = min(the k2-th smallest seed distance, the largest re-scored distance
// of the previous picks when there are k2 of them); the key holds T raised
// by one ulp with no window, so every window at distance <= T passes the
// bounds and is collected (report_window appends keys below it).
__global__ void __launch_bounds__(kSelThreads)
topk_threshold_kernel(const float* __restrict__ sd, int nseg, const float* __restrict__ prev_d,
                      const int* __restrict__ prev_n, int k2, unsigned long long* __restrict__ key,
                      float* __restrict__ t_out) {
    __shared__ int hist[256];
    __shared__ unsigned pfx;
    __shared__ unsigned pmax;  // float bits (distances are >= 0)
    float T = CDTW_INF;
    if (nseg >= k2) T = select_rank_f32(sd, nseg, k2 - 1, hist, &pfx);
    if (threadIdx.x == 0) pmax = 0u;
    __syncthreads();
    const bool have_prev = prev_n && *prev_n >= k2;
    if (have_prev) {
        unsigned m = 0u;
        for (int i = threadIdx.x; i < k2; i += blockDim.x) m = max(m, __float_as_uint(prev_d[i]));
        m = __reduce_max_sync(0xffffffffu, m);
        if ((threadIdx.x & 31) == 0) atomicMax(&pmax, m);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (have_prev) T = fminf(T, __uint_as_float(pmax));
        *t_out = T;
        *key = (T < CDTW_INF) ? pack_key(nextafterf(T, CDTW_INF), 0xffffffffu) : ~0ull;
    }
}

// Does window w overlap an accepted window?  acc[b + 1]: the accepted
// window of bucket b (starts bM .. bM + M - 1), or -1.
__device__ __forceinline__ bool overlaps_accepted(const int* acc, int w, int M) {
    const int b = w / M;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const int a = *(const volatile int*)(acc + b + d);  // buckets b-1, b, b+1
        if (a >= 0 && abs(a - w) < M) return true;
    }
    return false;
}

__global__ void __launch_bounds__(kSelThreads)
topk_greedy_kernel(const unsigned long long* __restrict__ hits, const int* __restrict__ nh_ptr,
                   int cap, int k2, int M, int* __restrict__ acc, int32_t* __restrict__ picks,
                   float* __restrict__ pick_d, int* __restrict__ npicks, int* __restrict__ status) {
    __shared__ unsigned long long keys[kGreedyB];
    __shared__ int hist[256];
    __shared__ int ulist[kSelThreads];
    __shared__ int wsum[kSelThreads / 32];
    __shared__ unsigned long long s_pfx;
    __shared__ int s_cnt, s_np, s_nu;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nh_all = *nh_ptr;
    if (nh_all > cap) {  // the hit list overflowed: no selection
        if (tid == 0) {
            *npicks = 0;
            *status = 1;
        }
        return;
    }
    const int nh = nh_all;
    if (tid == 0) {
        s_np = 0;
        *status = 0;
    }
    __syncthreads();
    unsigned long long lo = 0;  // keys below lo are consumed
    int consumed = 0;
    while (consumed < nh && s_np < k2) {
        const int take = min(kGreedyB, nh - consumed);
        // hi = the take-th smallest key >= lo (all of them when they fit)
        unsigned long long hi = ~0ull;
        if (take < nh - consumed) {
            unsigned long long prefix = 0, mask = 0;
            int r = take - 1;
            for (int shift = 56; shift >= 0; shift -= 8) {
                for (int d = tid; d < 256; d += kSelThreads) hist[d] = 0;
                __syncthreads();
                for (int i = tid; i < nh; i += kSelThreads) {
                    const unsigned long long k = hits[i];
                    if (k >= lo && (k & mask) == prefix)
                        atomicAdd(&hist[(unsigned)(k >> shift) & 255u], 1);
                }
                __syncthreads();
                if (tid == 0) s_pfx = prefix | ((unsigned long long)pick_digit(hist, &r) << shift);
                __syncthreads();
                prefix = s_pfx;
                mask |= 255ull << shift;
                __syncthreads();
            }
            hi = prefix;
        }
        // gather the keys in [lo, hi] (exactly `take`, keys are unique), sort
        if (tid == 0) s_cnt = 0;
        __syncthreads();
        for (int i = tid; i < nh; i += kSelThreads) {
            const unsigned long long k = hits[i];
            if (k >= lo && k <= hi) {
                const int at = atomicAdd(&s_cnt, 1);
                if (at < kGreedyB) keys[at] = k;
            }
        }
        __syncthreads();
        const int cnt = min(s_cnt, kGreedyB);
        int n2 = 1;
        while (n2 < cnt) n2 <<= 1;
        for (int i = cnt + tid; i < n2; i += kSelThreads) keys[i] = ~0ull;
        __syncthreads();
        for (int size = 2; size <= n2; size <<= 1) {
            for (int stride = size >> 1; stride > 0; stride >>= 1) {
                for (int t = tid; t < (n2 >> 1); t += kSelThreads) {
                    const int i = 2 * t - (t & (stride - 1));
                    const int j = i + stride;
                    const bool up = (i & size) == 0;
                    const unsigned long long a = keys[i], b = keys[j];
                    if ((a > b) == up) {
                        keys[i] = b;
                        keys[j] = a;
                    }
                }
                __syncthreads();
            }
        }
        // greedy over the ordered keys, kSelThreads at a time
        for (int base = 0; base < cnt && s_np < k2; base += kSelThreads) {
            const int i = base + tid;
            const bool valid = i < cnt;
            const int w = valid ? (int)(uint32_t)keys[i] : 0;
            const bool open = valid && !overlaps_accepted(acc, w, M);
            // ordered compaction of the open keys
            const unsigned bal = __ballot_sync(0xffffffffu, open);
            if (lane == 0) wsum[warp] = __popc(bal);
            __syncthreads();
            if (warp == 0) {
                const int c = wsum[lane];
                int incl = c;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int t = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += t;
                }
                wsum[lane] = incl - c;
                if (lane == 31) s_nu = incl;
            }
            __syncthreads();
            if (open) ulist[wsum[warp] + __popc(bal & ((1u << lane) - 1))] = i;
            __syncthreads();
            if (warp == 0) {
                const int nu = s_nu;
                int np = s_np;
                for (int c0 = 0; c0 < nu && np < k2; c0 += 32) {
                    const int j = c0 + lane;
                    const bool have = j < nu;
                    const int ki = have ? ulist[j] : 0;
                    const int wj = have ? (int)(uint32_t)keys[ki] : 0;
                    // earlier chunks of this round may have accepted a neighbour
                    unsigned m = __ballot_sync(0xffffffffu, have && !overlaps_accepted(acc, wj, M));
                    while (m && np < k2) {
                        const int src = __ffs(m) - 1;
                        const int wa = __shfl_sync(0xffffffffu, wj, src);
                        const int ka = __shfl_sync(0xffffffffu, ki, src);
                        if (lane == 0) {
                            acc[wa / M + 1] = wa;
                            picks[np] = wa;
                            pick_d[np] = key_dist(keys[ka]);
                        }
                        ++np;
                        m &= ~(1u << src);
                        m &= ~__ballot_sync(0xffffffffu, have && abs(wj - wa) < M);
                    }
                    __syncwarp();
                }
                if (lane == 0) s_np = np;
            }
            __syncthreads();
        }
        consumed += take;
        lo = hi + 1;
        __syncthreads();
    }
    if (tid == 0) *npicks = s_np;
}

}  // namespace

int launch_topk_threshold(cdtw_handle h, const float* sd, int nseg, const float* prev_d,
                          const int* prev_n, int k2, unsigned long long* key, float* t_out) {
    topk_threshold_kernel<<<1, kSelThreads, 0, h->stream>>>(sd, nseg, prev_d, prev_n, k2, key,
                                                           t_out);
    CDTW_LAUNCH(h, "topk_threshold_kernel");
    return CDTW_OK;
}

int launch_topk_greedy(cdtw_handle h, const unsigned long long* hits, const int* nh, int cap,
                       int k2, int M, int* acc, int32_t* picks, float* pick_d, int* npicks,
                       int* status) {
    topk_greedy_kernel<<<1, kSelThreads, 0, h->stream>>>(hits, nh, cap, k2, M, acc, picks, pick_d,
                                                        npicks, status);
    CDTW_LAUNCH(h, "topk_greedy_kernel");
    return CDTW_OK;
}

}  // namespace cdtw
