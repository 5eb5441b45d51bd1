// Differentiable pairwise cDTW: z-normalisation, backward kernels and the
// host launchers.  The forward device code and its description are in
// pair.cuh (instantiated in pair_part0..3.cu).
#include "pair.cuh"

#include <algorithm>

namespace cdtw {

namespace {

// z-normalisation of every series of the pairs: one warp per series, FP64
// two-pass mean / population variance (sigma = 1 when var <= 0, flagged by a
// negative sigma in the header), z written as float.
__global__ void pair_znorm_kernel(const float* __restrict__ q, const float* __restrict__ s,
                                  int64_t n, int L, float* __restrict__ zq,
                                  float* __restrict__ zs, double* __restrict__ hdr) {
    const int lane = threadIdx.x & 31;
    const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (wid >= 2 * n) return;
    const int64_t pr = wid >> 1;
    const bool isq = (wid & 1) == 0;
    const float* x = (isq ? q : s) + pr * L;
    float* z = (isq ? zq : zs) + pr * L;
    double s1 = 0.0;
    for (int t = lane; t < L; t += 32) s1 += (double)__ldg(x + t);
    for (int o = 16; o > 0; o >>= 1) s1 += __shfl_xor_sync(kFull, s1, o);
    const double mu = s1 / (double)L;
    double s2 = 0.0;
    for (int t = lane; t < L; t += 32) {
        const double v = (double)__ldg(x + t) - mu;
        s2 = fma(v, v, s2);
    }
    for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(kFull, s2, o);
    const double var = s2 / (double)L;
    const double sd = var > 0.0 ? sqrt(var) : 1.0;
    const double inv = 1.0 / sd;
    for (int t = lane; t < L; t += 32) z[t] = pair_z(__ldg(x + t), mu, inv);
    if (hdr && lane == 0) {
        hdr[pr * 4 + (isq ? 0 : 2)] = mu;
        hdr[pr * 4 + (isq ? 1 : 3)] = var > 0.0 ? sd : -1.0;
    }
}

constexpr int kBwdThreads = 128;

// Block-wide FP64 sums of a and b (every thread gets them); blocks of 1 to 4
// warps; red holds 2 x 4 doubles.
__device__ __forceinline__ void block_sum2(double& a, double& b, double* red) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(kFull, a, o);
        b += __shfl_xor_sync(kFull, b, o);
    }
    __syncthreads();  // red may still be read from a previous call
    if (lane == 0) {
        red[wid] = a;
        red[4 + wid] = b;
    }
    __syncthreads();
    const int nw = blockDim.x >> 5;
    a = 0.0;
    b = 0.0;
    for (int w = 0; w < nw; ++w) {
        a += red[w];
        b += red[4 + w];
    }
}

// The same by one warp (lane slices, warp scan of the slice totals).
__device__ void warp_prefix(const float* x, double* P, int L, int lane) {
    const int per = (L + 31) / 32;
    const int lo = min(lane * per, L), hi = min(lo + per, L);
    double tot = 0.0;
    for (int t = lo; t < hi; ++t) tot += (double)x[t];
    double inc = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double v = __shfl_up_sync(kFull, inc, o);
        if (lane >= o) inc += v;
    }
    double run = inc - tot;
    for (int t = lo; t < hi; ++t) {
        P[t] = run;
        run += (double)x[t];
    }
    if (lane == 31) P[L] = inc;
    __syncwarp();
}

// Exclusive FP64 prefix sums P[0..L] of the L floats in x by the block: each
// thread a contiguous slice, a scan of the slice totals across the block.
__device__ void block_prefix(const float* x, double* P, int L, double* red) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nt = blockDim.x;
    const int per = (L + nt - 1) / nt;
    const int lo = min((int)threadIdx.x * per, L), hi = min(lo + per, L);
    double tot = 0.0;
    for (int t = lo; t < hi; ++t) tot += (double)x[t];
    double inc = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double v = __shfl_up_sync(kFull, inc, o);
        if (lane >= o) inc += v;
    }
    __syncthreads();
    if (lane == 31) red[wid] = inc;
    __syncthreads();
    double base = 0.0;
    for (int w = 0; w < wid; ++w) base += red[w];
    double run = base + inc - tot;
    for (int t = lo; t < hi; ++t) {
        P[t] = run;
        run += (double)x[t];
    }
    if ((int)threadIdx.x == nt - 1) P[L] = base + inc;
    __syncthreads();
}

// Backward, one pair per scope: a warp (BLOCK = false, several pairs per
// block, L <= 1024) or the whole block (BLOCK = true, four warps, longer
// series); the pair's z values staged in shared memory.  g_q[i] = sum over the
// row run [a_i, b_i] of f'(zq_i - zs_j), g_s[j] = -sum over the column run;
// then through the z-normalisation and scaled by dD.  For the squared cost
// f'(d) = 2d and a run sum is 2 (len zq_i - (P[b+1] - P[a])) with FP64 prefix
// sums P of the other series: no per-run loop.  Runs are clamped to
// [0, L-1], so a damaged path record cannot index outside the staged series.
template <bool EU, bool BLOCK>
__global__ void __launch_bounds__(kBwdThreads)
pair_bwd_kernel(const float* __restrict__ q, const float* __restrict__ s, int64_t n, int L,
                const double* __restrict__ hdr, const uint32_t* __restrict__ rows,
                const uint32_t* __restrict__ cols, const float* __restrict__ dD,
                float* __restrict__ dq, float* __restrict__ ds) {
    extern __shared__ __align__(16) unsigned char bsm[];
    __shared__ double red[8];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int64_t pr = BLOCK ? (int64_t)blockIdx.x : (int64_t)blockIdx.x * (blockDim.x >> 5) + wid;
    if (pr >= n) return;  // whole scope
    const int me = BLOCK ? (int)threadIdx.x : lane;
    const int step = BLOCK ? (int)blockDim.x : 32;
    auto sync = [] {
        if (BLOCK) __syncthreads();
        else __syncwarp();
    };
    const size_t wbytes = (size_t)round_up((int64_t)((EU ? 8 * (size_t)(L + 1) : 0) + 8 * (size_t)L), 16);
    double* P = (double*)(bsm + (BLOCK ? 0 : (size_t)wid * wbytes));  // L + 1 (squared cost)
    float* zqs = (float*)(P + (EU ? L + 1 : 0));
    float* zss = zqs + L;
    const bool zn = hdr != nullptr;
    double muq = 0.0, invq = 1.0, mus = 0.0, invs = 1.0;
    bool degq = false, degs = false;
    if (zn) {
        muq = hdr[pr * 4 + 0];
        const double sdq = hdr[pr * 4 + 1];
        mus = hdr[pr * 4 + 2];
        const double sds = hdr[pr * 4 + 3];
        degq = sdq < 0.0;
        degs = sds < 0.0;
        invq = 1.0 / (degq ? 1.0 : sdq);
        invs = 1.0 / (degs ? 1.0 : sds);
    }
    const float* xq = q + pr * L;
    const float* xs = s + pr * L;
    for (int t = me; t < L; t += step) {
        const float a = __ldg(xq + t), b = __ldg(xs + t);
        zqs[t] = zn ? pair_z(a, muq, invq) : a;
        zss[t] = zn ? pair_z(b, mus, invs) : b;
    }
    sync();
    auto fp = [](float df) { return df > 0.f ? 1.0f : (df < 0.f ? -1.0f : 0.0f); };
    const float up = dD ? __ldg(dD + pr) : 1.0f;
    for (int side = 0; side < 2; ++side) {
        float* out = side == 0 ? dq : ds;
        if (!out) continue;
        out += pr * L;
        const uint32_t* run = (side == 0 ? rows : cols) + pr * L;
        const float* zt_s = side == 0 ? zqs : zss;
        const float* zo_s = side == 0 ? zss : zqs;
        if (EU) {
            if (BLOCK) block_prefix(zo_s, P, L, red);
            else warp_prefix(zo_s, P, L, lane);
        }
        double sg = 0.0, sgz = 0.0;
        for (int t = me; t < L; t += step) {
            const uint32_t r = __ldg(run + t);
            const int hi = min((int)(r >> 16), L - 1);
            const int lo = min((int)(r & 0xffffu), hi);
            const float zt = zt_s[t];
            float g;
            if (EU) {
                // q side: sum_j 2 (zq_t - zs_j); s side: -sum_i 2 (zq_i - zs_t)
                // = sum_i 2 (zs_t - zq_i): both 2 (len z_t - sum of the other)
                const double sum = (double)(hi - lo + 1) * (double)zt - (P[hi + 1] - P[lo]);
                g = (float)(2.0 * sum);
            } else {
                g = 0.f;
                for (int u = lo; u <= hi; ++u) {
                    const float o = zo_s[u];
                    g += side == 0 ? fp(__fsub_rn(zt, o)) : -fp(__fsub_rn(o, zt));
                }
            }
            out[t] = zn ? g : g * up;
            sg += (double)g;
            sgz += (double)g * (double)zt;
        }
        if (zn) {
            if (BLOCK) {
                block_sum2(sg, sgz, red);
            } else {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    sg += __shfl_xor_sync(kFull, sg, o);
                    sgz += __shfl_xor_sync(kFull, sgz, o);
                }
            }
            const bool deg = side == 0 ? degq : degs;
            const double inv = side == 0 ? invq : invs;
            const double mg = sg / (double)L, mgz = deg ? 0.0 : sgz / (double)L;
            for (int t = me; t < L; t += step)  // each thread re-reads its own values
                out[t] = (float)((double)up * ((double)out[t] - mg - (double)zt_s[t] * mgz) * inv);
        }
        sync();  // P is rebuilt for the other side
    }
}

PairFwdK fwd_kernel(int C, bool eu, int dm) {
    if (C <= 4) return pair_fwd_part0(C, eu, dm);
    if (C <= 8) return pair_fwd_part1(C, eu, dm);
    if (C <= 12) return pair_fwd_part2(C, eu, dm);
    return pair_fwd_part3(C, eu, dm);
}

}  // namespace

// Lanes per pair (G, a power of two) and band slots per lane (C): about four
// cells per lane for short bands, 32 lanes for long ones.
void pair_shape(int L, int W, int* G, int* C) {
    (void)L;
    const int slots = W + 1;
    int g = 1;
    while (g < 32 && (slots + g - 1) / g > 4) g *= 2;
    *G = g;
    *C = (slots + g - 1) / g;
}

// Shared-record mode of the forward with a path: the record stays in shared
// memory when it takes at most 512 bytes per lane (C <= 4, one byte per lane
// and anti-diagonal) and the block's records and move logs leave room for 3
// blocks per SM.  recb / logb: bytes per group, with strides of 32 (mod 128)
// bytes so the groups of a warp sit on different shared-memory banks.
static bool pair_shared_record(int L, int G, int C, int* recb, int* logb, size_t* bytes) {
    const int K = 2 * L - 1;
    *recb = (int)round_up((int64_t)K * G, 128) + 32;
    *logb = (int)round_up(K, 128) + 32;
    *bytes = (size_t)(kPairThreads / G) * (size_t)(*recb + *logb);
    return C <= 4 && K <= 512 && *bytes <= kSharedRecMax;
}

// Words of direction record per pair in device scratch: whole backtracking
// chunks of R anti-diagonals x G lane elements; 0 in shared-record mode.
size_t pair_dirs_words(int L, int W) {
    int G, C;
    pair_shape(L, W, &G, &C);
    int recb, logb;
    size_t shared_bytes;
    if (pair_shared_record(L, G, C, &recb, &logb, &shared_bytes)) return 0;
    const int eb = C <= 4 ? 1 : (C <= 8 ? 2 : 4);
    const int64_t nch = div_up(2 * (int64_t)L - 1, kWalkChunk / eb);
    return (size_t)(nch * kWalkChunk * G / 4);
}

// Checkpointed mode: anti-diagonals per segment (a multiple of 2C, about
// 128) and segments per pair (segment 0 also covers the first one or two
// steps before the bodies).
static int pair_ckpt_seg(int C) { return 2 * C * std::max(2, 128 / (2 * C)); }

static int pair_ckpt_nseg(int L, int W, int C) {
    const int K = 2 * L - 1, k0 = (W & 1) ? 2 : 1;
    return (int)std::max<int64_t>(1, div_up(std::max(K - k0, 1), pair_ckpt_seg(C)));
}

// Floats of checkpoints per pair in device scratch (two anti-diagonals of
// G x C slots per segment); 0 where the pair runs in shared-record mode.
size_t pair_ckpt_floats(int L, int W) {
    int G, C;
    pair_shape(L, W, &G, &C);
    int recb, logb;
    size_t shared_bytes;
    if (C < 2 || pair_shared_record(L, G, C, &recb, &logb, &shared_bytes)) return 0;
    return (size_t)pair_ckpt_nseg(L, W, C) * 2 * C * G;
}

int launch_pair_znorm(cdtw_handle h, const float* q, const float* s, int64_t n, int L, float* zq,
                      float* zs, double* hdr) {
    const int64_t warps = 2 * n;
    const int blocks = (int)div_up(warps * 32, 256);
    pair_znorm_kernel<<<blocks, 256, 0, h->stream>>>(q, s, n, L, zq, zs, hdr);
    CDTW_LAUNCH(h, "pair_znorm_kernel");
    return CDTW_OK;
}

int launch_pair_fwd(cdtw_handle h, const float* zq, const float* zs, int64_t n, int L, int W,
                    bool euclid, float* D, uint32_t* dirs, uint32_t* rows, uint32_t* cols,
                    int64_t qstride, const int* gate, int gate_max, int gate_min,
                    bool wide) {
    int G, C;
    pair_shape(L, W, &G, &C);
    if (C > 16) return set_error(h, CDTW_EUNSUPPORTED, "pair band W=%d exceeds 511", W);
    if (!rows && wide) {
        G = 32;
        C = (W + 1 + G - 1) / G;
    } else if (!rows && G > 4 && (W + 1 + G / 2 - 1) / (G / 2) <= 8) {
        // distance only (no record whose layout fixes the shape): half as
        // many lanes with twice the cells each -- more independent cells per
        // step for the same dependent chain (measured: the search's seed pass
        // at M=512, W=51 120 -> 105 us; wider groups were slower)
        G /= 2;
        C = (W + 1 + G - 1) / G;
    }
    PairArgs a;
    a.zq = zq;
    a.zs = zs;
    a.qstride = qstride < 0 ? L : qstride;
    a.gate = gate;
    a.gate_max = gate_max;
    a.gate_min = gate_min;
    a.n = n;
    a.L = L;
    a.W = W;
    a.G = G;
    a.lgG = 0;
    while ((1 << a.lgG) < G) ++a.lgG;
    a.D = D;
    a.dirs = dirs;
    a.dstride = (int)pair_dirs_words(L, W);
    a.rows = rows;
    a.cols = cols;
    a.ckpt = nullptr;
    a.seg = 0;
    a.nseg = 0;
    const int threads = kPairThreads;
    const int64_t groups_per_block = threads / G;
    // a path is recorded when the run arrays are given; the direction scratch
    // is needed only outside shared-record mode
    size_t shared_rec;
    const bool shared = pair_shared_record(L, G, C, &a.recb, &a.logb, &shared_rec);
    const int dm = !rows ? 0 : shared ? 2 : 1;
    if (dm != 0 && !cols) return set_error(h, CDTW_EINVAL, "path record without column runs");
    if (dm == 1 && !dirs) return set_error(h, CDTW_EINVAL, "path record without direction scratch");
    // DM 1: backtracking ring (kWalkStages chunks of kWalkChunk bytes per lane)
    // + move log per group
    const size_t smem =
        dm == 2   ? shared_rec
        : dm == 1 ? (size_t)threads * kWalkStages * kWalkChunk + (size_t)groups_per_block * kMoveLog
                  : 0;
    const int64_t blocks = div_up(n, groups_per_block);
    if (blocks > INT32_MAX) return set_error(h, CDTW_EINVAL, "too many pairs");
    const PairFwdK k = fwd_kernel(C, euclid, dm);
    CDTW_CUDA(h, cudaFuncSetAttribute((const void*)k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
    k<<<(int)blocks, threads, smem, h->stream>>>(a);
    CDTW_LAUNCH(h, "pair_fwd_kernel");
    return CDTW_OK;
}

// Checkpointed path record: the forward without direction bits storing
// checkpoints every pair_ckpt_seg anti-diagonals, then the segment-wise
// recomputation and walk (pair_ckpt_walk_kernel) writing the row and column
// runs.  Needs C >= 2 outside shared-record mode (pair_ckpt_floats > 0).
int launch_pair_fwd_ckpt(cdtw_handle h, const float* zq, const float* zs, int64_t n, int L,
                         int W, bool euclid, float* D, float* ckpt, uint32_t* rows,
                         uint32_t* cols) {
    if (pair_ckpt_floats(L, W) == 0)
        return set_error(h, CDTW_EUNSUPPORTED, "no checkpointed mode for L=%d W=%d", L, W);
    int G, C;
    pair_shape(L, W, &G, &C);
    PairArgs a;
    a.zq = zq;
    a.zs = zs;
    a.qstride = L;
    a.gate = nullptr;
    a.gate_max = 0;
    a.gate_min = -1;
    a.n = n;
    a.L = L;
    a.W = W;
    a.G = G;
    a.lgG = 0;
    while ((1 << a.lgG) < G) ++a.lgG;
    a.D = D;
    a.dirs = nullptr;
    a.dstride = 0;
    a.rows = rows;
    a.cols = cols;
    a.ckpt = ckpt;
    a.seg = pair_ckpt_seg(C);
    a.nseg = pair_ckpt_nseg(L, W, C);
    const int threads = kPairThreads;
    const int64_t groups_per_block = threads / G;
    const int64_t blocks = div_up(n, groups_per_block);
    if (blocks > INT32_MAX) return set_error(h, CDTW_EINVAL, "too many pairs");
    const int eb = C <= 4 ? 1 : (C <= 8 ? 2 : 4);
    // records of the longest segment (segment 0 holds up to seg + 2 rows)
    a.recb = (int)round_up((int64_t)(a.seg + 2) * G * eb, 128) + 32;
    a.logb = (int)round_up(a.seg + 2, 128) + 32;
    const PairFwdK kf = fwd_kernel(C, euclid, 3);
    kf<<<(int)blocks, threads, 0, h->stream>>>(a);
    CDTW_LAUNCH(h, "pair_fwd_kernel");
    const PairFwdK kw = fwd_kernel(C, euclid, 4);
    const size_t smem = (size_t)groups_per_block * (size_t)(a.recb + a.logb);
    CDTW_CUDA(h, cudaFuncSetAttribute((const void*)kw, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
    kw<<<(int)blocks, threads, smem, h->stream>>>(a);
    CDTW_LAUNCH(h, "pair_ckpt_walk_kernel");
    return CDTW_OK;
}

int launch_pair_bwd(cdtw_handle h, const float* q, const float* s, int64_t n, int L,
                    const double* hdr, const uint32_t* rows, const uint32_t* cols,
                    const float* dD, bool euclid, float* dq, float* ds) {
    // per pair: z of both series (8L bytes) and, for the squared cost, one
    // prefix-sum array (8(L+1) bytes); a warp per pair (up to 4 per block,
    // 96 KB) for L <= 1024, a 4-warp block per pair above
    const size_t wbytes =
        (size_t)round_up((int64_t)((euclid ? 8 * (size_t)(L + 1) : 0) + 8 * (size_t)L), 16);
    const bool block = L > 1024;
    const int nw = block ? 1 : (int)std::max<size_t>(1, std::min<size_t>(4, 96 * 1024 / wbytes));
    const size_t smem = block ? wbytes : (size_t)nw * wbytes;
    const int64_t blocks = block ? n : div_up(n, nw);
    if (blocks > INT32_MAX) return set_error(h, CDTW_EINVAL, "too many pairs");
    auto k = euclid ? (block ? pair_bwd_kernel<true, true> : pair_bwd_kernel<true, false>)
                    : (block ? pair_bwd_kernel<false, true> : pair_bwd_kernel<false, false>);
    CDTW_CUDA(h, cudaFuncSetAttribute((const void*)k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
    k<<<(unsigned)blocks, block ? kBwdThreads : nw * 32, smem, h->stream>>>(q, s, n, L, hdr, rows,
                                                                           cols, dD, dq, ds);
    CDTW_LAUNCH(h, "pair_bwd_kernel");
    return CDTW_OK;
}

}  // namespace cdtw
