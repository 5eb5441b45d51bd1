// Lane-block kernels (band spread over a group of lanes, two windows per
// group): shape choice and launchers for all listed windows and for the
// single-query search.  The device code and its description are in
// cdtw_lane.cuh.
#include "cdtw_lane.cuh"

#include <algorithm>
#include <mutex>

namespace cdtw {

namespace {

struct LaneKernels {
    LaneKernel eu[kLaneBMax + 1] = {};
    LaneKernel mh[kLaneBMax + 1] = {};
    LaneKernel seu[kLaneBMax + 1] = {};
    LaneKernel smh[kLaneBMax + 1] = {};
    LaneKernels() {
        lane_fill_part0(eu, mh, seu, smh);
        lane_fill_part1(eu, mh, seu, smh);
        lane_fill_part2(eu, mh, seu, smh);
        lane_fill_part3(eu, mh, seu, smh);
    }
};

const LaneKernels& lane_kernels() {
    static LaneKernels k;
    return k;
}

// Float4s between the starts of consecutive query copies in shared memory
// (the copy rounded up to 8 float4s, plus 8 for the bank offsets below).
int lane_copy_stride(const QueryPack& q) { return (q.lq / 4 + 7) / 8 * 8 + 8; }

// Shared-memory bytes of the query copies the kernels stage per block.
size_t lane_smem(const QueryPack& q) {
    return (size_t)4 * lane_copy_stride(q) * sizeof(float4);
}

// Bank offsets of the query copies.  At step t lane g of a group reads the
// float4s b >> 2, (b >> 2) + 1, ... of copy b & 3, b = t + g (B-1).  Eight
// lanes' 16-byte reads (a quarter warp) are served in one shared-memory
// wavefront when their float4 indices differ mod 8, so copy c is placed at
// c * stride + e[c] (stride a multiple of 8) with e[c] in [0, 8) chosen to
// minimise the wavefronts of the reads over the 32-step period of the
// pattern (the groups of a warp read the same addresses; e[0] = 0).  With the
// copies back to back the reads of a wide band took up to 11 wavefronts per
// instruction against 4 at best.
void lane_copy_offsets(int B, int G, int e[4]) {
    static std::mutex mu;
    static bool done[kLaneBMax + 1][6] = {};
    static int table[kLaneBMax + 1][6][4];
    int lg = 0;
    while ((1 << lg) < G) ++lg;
    std::lock_guard<std::mutex> lock(mu);
    if (!done[B][lg]) {
        const int D = B - 1;
        long best = -1;
        int be[4] = {0, 0, 0, 0};
        for (int e1 = 0; e1 < 8; ++e1)
            for (int e2 = 0; e2 < 8; ++e2)
                for (int e3 = 0; e3 < 8; ++e3) {
                    const int off[4] = {0, e1, e2, e3};
                    long cost = 0;
                    for (int t = 0; t < 32; ++t)
                        for (int qw = 0; qw < 4; ++qw) {
                            int idx[8];
                            int n = 0;
                            for (int lane = 8 * qw; lane < 8 * qw + 8; ++lane) {
                                const int b = t + (lane & (G - 1)) * D;
                                const int v = off[b & 3] + (b >> 2);
                                bool seen = false;
                                for (int i = 0; i < n; ++i) seen = seen || idx[i] == v;
                                if (!seen) idx[n++] = v;
                            }
                            int per[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                            int worst = 0;
                            for (int i = 0; i < n; ++i) worst = std::max(worst, ++per[idx[i] & 7]);
                            cost += worst;
                        }
                    if (best < 0 || cost < best) {
                        best = cost;
                        be[1] = e1;
                        be[2] = e2;
                        be[3] = e3;
                    }
                }
        for (int c = 0; c < 4; ++c) table[B][lg][c] = be[c];
        done[B][lg] = true;
    }
    for (int c = 0; c < 4; ++c) e[c] = table[B][lg][c];
}

int fill_lane_args(cdtw_handle h, const float* x, int64_t N, const double* mu,
                   const float* sigma, LaneArgs* a) {
    const QueryPack& q = h->q;
    int G, B;
    if (!lane_shape(q.W, &G, &B))
        return set_error(h, CDTW_EUNSUPPORTED, "band W=%d outside the lane-block kernels", q.W);
    if (q.lq < lane_qpad_min(q.M, q.W))
        return set_error(h, CDTW_EUNSUPPORTED, "query pack too short for the lane-block kernels");
    a->x = x;
    a->mu = mu;
    a->sigma = sigma;
    a->qpad4 = (const float4*)q.qpad;
    a->lq4 = q.lq / 4;
    // one group per warp (G = 32): the reads of the 32 lanes are all
    // distinct and shared memory limits the kernel, so the copies take the
    // bank offsets that spread them; narrower groups read each address twice
    // or more and keep the copies back to back (measured: the offsets gave
    // +16 % at W = 409, -2 % at W = 102 and 204)
    int e[4] = {0, 0, 0, 0};
    if (G == 32) lane_copy_offsets(B, G, e);
    const int stride = G == 32 ? lane_copy_stride(q) : a->lq4;
    for (int c = 0; c < 4; ++c) a->qoff[c] = c * stride + e[c];
    a->qenv = q.env;
    a->M = q.M;
    a->W = q.W;
    a->G = G;
    a->lgG = 0;
    while ((1 << a->lgG) < G) ++a->lgG;
    a->Nw = (int)(N - q.M + 1);
    a->gW = q.W / B;
    a->cW = q.W % B;
    a->cph = 2 * q.W + 1 - (G - 1) * B;
    a->idx = nullptr;
    a->L = 0;
    a->out = nullptr;
    a->cands = nullptr;
    a->count = nullptr;
    a->work = nullptr;
    a->key = nullptr;
    return CDTW_OK;
}

}  // namespace

// Lanes per window group (G, a power of two) and cells per lane (B) for band
// W: every B in [kLaneBMin, kLaneBMax] and G in {4, 8, 16, 32} with
// G*B >= 2W+1 and (G-1)*B <= 2W (the cells past the band, k > 2W, all lie in
// lane G-1 and k = 2W+1 is not its slot 0), at the least estimated issue cost
// per row: 3 instructions per cell and about 10 per lane and window of row
// overhead.  False when none fits.
bool lane_shape(int W, int* G, int* B) {
    const int cells = 2 * W + 1;
    long best = -1;
    for (int g = 4; g <= 32; g *= 2) {
        for (int b = kLaneBMin; b <= kLaneBMax; ++b) {
            if ((long)g * b < cells || (long)(g - 1) * b > 2L * W) continue;
            const long cost = 3L * g * b + 10L * g;
            if (best < 0 || cost < best) {
                best = cost;
                *G = g;
                *B = b;
            }
        }
    }
    return best >= 0;
}

int lane_qpad_min(int M, int W) { return M + 2 * W + 52; }

int launch_cdtw_lane(cdtw_handle h, const float* x, int64_t N, const double* mu,
                     const float* sigma, const int32_t* idx, int64_t L, bool euclid,
                     float* out) {
    if (L <= 0) return CDTW_OK;
    LaneArgs a;
    CDTW_TRY(fill_lane_args(h, x, N, mu, sigma, &a));
    int G, B;
    lane_shape(h->q.W, &G, &B);
    a.idx = idx;
    a.L = (int)L;
    a.out = out;
    const LaneKernel k = euclid ? lane_kernels().eu[B] : lane_kernels().mh[B];
    const size_t smem = lane_smem(h->q);
    CDTW_CUDA(h, cudaFuncSetAttribute((const void*)k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
    const int64_t units = div_up(L, 2);
    const int64_t per_block = kLaneThreads / G;
    const int64_t blocks = div_up(units, per_block);
    if (blocks > INT32_MAX) return set_error(h, CDTW_EINVAL, "too many windows");
    k<<<(unsigned)blocks, kLaneThreads, smem, h->stream>>>(a);
    CDTW_LAUNCH(h, "cdtw_lane_kernel");
    return CDTW_OK;
}

int launch_cdtw_lane_search(cdtw_handle h, const float* x, int64_t N, const double* mu,
                            const float* sigma, const Cand* cands, const int* count, int* work,
                            int max_count, bool euclid, unsigned long long* key,
                            const HitSink& sink) {
    if (max_count <= 0) return CDTW_OK;
    LaneArgs a;
    CDTW_TRY(fill_lane_args(h, x, N, mu, sigma, &a));
    int G, B;
    lane_shape(h->q.W, &G, &B);
    a.cands = cands;
    a.count = count;
    a.work = work;
    a.key = key;
    a.sink = sink;
    const LaneKernel k = euclid ? lane_kernels().seu[B] : lane_kernels().smh[B];
    const size_t smem = lane_smem(h->q);
    CDTW_CUDA(h, cudaFuncSetAttribute((const void*)k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
    int per_sm = 0;
    CDTW_CUDA(h, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)k,
                                                               kLaneThreads, smem));
    const int64_t per_block = (int64_t)(kLaneThreads / 32) * (64 / G);  // candidates per round
    const int64_t want = div_up(max_count, per_block);
    const unsigned blocks = (unsigned)std::max<int64_t>(
        1, std::min<int64_t>(want, (int64_t)std::max(per_sm, 1) * h->sm_count));
    k<<<blocks, kLaneThreads, smem, h->stream>>>(a);
    CDTW_LAUNCH(h, "cdtw_lane_search_kernel");
    return CDTW_OK;
}

}  // namespace cdtw
