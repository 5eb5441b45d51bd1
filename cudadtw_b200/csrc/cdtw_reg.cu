// Banded DTW with the whole band of one window in registers ("register band").
//
// Reference: sparse_block_cdtw / dense_block_cdtw (include/cdtw.cuh:164-363),
// which spread one window over W+2 threads and step the anti-diagonals through
// shared memory with a __syncthreads per step.  Windows are independent and
// there are millions of them, so here one thread owns one window and keeps
// the 2W+1 band cells of the current row in registers; the 32 lanes of a warp
// run 32 neighbouring windows in lockstep, so all lanes read the same query
// values (a shared-memory broadcast) and consecutive stream samples (one
// coalesced 128-byte load per row).
//
// Orientation: rows are window (data) positions j = 0..M-1, columns are query
// positions i, band coordinate k = i - j + W in [0, 2W].  The cell update
//   D[j][k] = cost(z_j, q_{j-W+k}) + min(D[j-1][k], D[j-1][k+1], D[j][k-1])
// is one FADD, one three-input FMNMX and one FFMA.  Query positions outside
// [0, M) are padded with +inf, which makes out-of-matrix cells +inf without
// any per-cell test.  The result D[M-1][W] equals the reference's
// penalty[...][M] (cdtw.cuh:83).
#include "cdtw_reg.cuh"

namespace cdtw {

namespace {

struct RegKernels {
    RegKernel eu[kMaxRegW + 1];
    RegKernel mh[kMaxRegW + 1];
    RegSearchKernel seu[kMaxRegW + 1];
    RegSearchKernel smh[kMaxRegW + 1];
    RegKernel eu2[kMaxReg2W + 1];  // two windows per thread
    RegKernel mh2[kMaxReg2W + 1];
    RegKernel eu4[kMaxReg4W + 1];  // four windows per thread
    RegKernel mh4[kMaxReg4W + 1];
    RegCKernel euc[kMaxReg2W + 1];  // consecutive windows, all of them
    RegCKernel mhc[kMaxReg2W + 1];
    RegKernels() {
        void** a = (void**)eu;
        void** b = (void**)mh;
        void** c = (void**)seu;
        void** d = (void**)smh;
        reg_fill_part0(a, b, c, d);
        reg_fill_part1(a, b, c, d);
        reg_fill_part2(a, b, c, d);
        reg_fill_part3(a, b, c, d);
        reg_fill_part4(a, b, c, d);
        reg_fill_part5(a, b, c, d);
        reg2_fill_part0((void**)eu2, (void**)mh2);
        reg2_fill_part1((void**)eu2, (void**)mh2);
        reg4_fill_part0((void**)eu4, (void**)mh4);
        regc_fill_part0((void**)euc, (void**)mhc);
        regc_fill_part1((void**)euc, (void**)mhc);
        regc_fill_part2((void**)euc, (void**)mhc);
    }
};

const RegKernels& reg_kernels() {
    static RegKernels k;
    return k;
}

}  // namespace

int max_register_band() { return kMaxRegW; }

int choose_variant(cdtw_handle h, int W) {
    int v = (W >= 0 && W < CDTW_MAX_QUERY) ? h->band_variant[W] : 0;
    int G, B;
    const bool lane = lane_shape(W, &G, &B) && h->q.lq >= lane_qpad_min(h->q.M, W);
    if (v == CDTW_VARIANT_REGISTER && W > kMaxRegW) v = 0;
    if (v == CDTW_VARIANT_STRIP16 && W < 15) v = 0;
    if (v == CDTW_VARIANT_STRIP32 && W < 31) v = 0;
    if (v == CDTW_VARIANT_LANE && !lane) v = 0;
    if (v == 0)
        v = (W <= kMaxRegW) ? CDTW_VARIANT_REGISTER
                            : (lane ? CDTW_VARIANT_LANE : CDTW_VARIANT_STRIP16);
    return v;
}

int launch_cdtw_strip_search(cdtw_handle h, const float* x, int64_t N, const double* mu,
                             const float* sigma, const Cand* cands, const int* count, int* work,
                             int max_count, bool euclid, int R, unsigned long long* key,
                             const HitSink& sink);

int launch_cdtw_search(cdtw_handle h, const float* x, int64_t N, const double* mu,
                       const float* sigma, const Cand* cands, const int* count, int* work,
                       int max_count, bool euclid, unsigned long long* key,
                       const HitSink& sink) {
    const QueryPack& q = h->q;
    if (max_count <= 0) return CDTW_OK;
    const int variant = choose_variant(h, q.W);
    if (variant == CDTW_VARIANT_LANE)
        return launch_cdtw_lane_search(h, x, N, mu, sigma, cands, count, work, max_count, euclid,
                                       key, sink);
    if (variant != CDTW_VARIANT_REGISTER)
        return launch_cdtw_strip_search(h, x, N, mu, sigma, cands, count, work, max_count,
                                        euclid, variant == CDTW_VARIANT_STRIP16 ? 16 : 32, key,
                                        sink);
    RegSearchKernel k = euclid ? reg_kernels().seu[q.W] : reg_kernels().smh[q.W];
    const int lq4 = q.lq / 4;
    const size_t smem = (size_t)q.lq * 4 * sizeof(float) + (size_t)q.M * sizeof(float2);
    CDTW_CUDA(h, cudaFuncSetAttribute((const void*)k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
    int per_sm = 0;
    CDTW_CUDA(h, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)k, kRegBlock,
                                                               smem));
    const int64_t want = div_up(max_count, kRegBlock);
    const unsigned blocks = (unsigned)std::max<int64_t>(
        1, std::min<int64_t>(want, (int64_t)std::max(per_sm, 1) * h->sm_count));
    k<<<blocks, kRegBlock, smem, h->stream>>>(x, mu, sigma, (const float4*)q.qpad, lq4, q.env,
                                              q.M, cands, count, work, key, sink);
    CDTW_LAUNCH(h, "cdtw_reg_search_kernel");
    return CDTW_OK;
}

int launch_cdtw_windows(cdtw_handle h, const float* x, int64_t N, const double* mu,
                        const float* sigma, const int32_t* idx, int64_t L, bool euclid,
                        float* out) {
    const QueryPack& q = h->q;
    const int Nw = (int)(N - q.M + 1);
    const int variant = q.qrev ? choose_variant(h, q.W) : CDTW_VARIANT_REGISTER;
    if (variant == CDTW_VARIANT_LANE)
        return launch_cdtw_lane(h, x, N, mu, sigma, idx, L, euclid, out);
    if (variant != CDTW_VARIANT_REGISTER || q.W > kMaxRegW) {
        if (!q.qrev)
            return set_error(h, CDTW_EUNSUPPORTED, "band W=%d above the register-band limit %d",
                             q.W, kMaxRegW);
        return launch_cdtw_strip(h, x, N, mu, sigma, idx, L, euclid,
                                 variant == CDTW_VARIANT_STRIP16 ? 16 : 32, out);
    }
    if (L <= 0) return CDTW_OK;
    // four windows per thread up to W = kMaxReg4W, two up to kMaxReg2W
    // (register budget)
    const int per = q.W <= kMaxReg4W ? 4 : (q.W <= kMaxReg2W ? 2 : 1);
    const int lq4 = q.lq / 4;
    const size_t smem = (size_t)q.lq * 4 * sizeof(float);
    if (!idx && per > 1 && L == Nw) {
        // every window: the consecutive-window kernels (one sliding run of
        // the stream per thread)
        RegCKernel kc = euclid ? reg_kernels().euc[q.W] : reg_kernels().mhc[q.W];
        if (smem > 48 * 1024)
            CDTW_CUDA(h, cudaFuncSetAttribute((const void*)kc,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)smem));
        const unsigned blocks =
            (unsigned)div_up(div_up(L, regc_per_thread(q.W)), kRegBlock);
        kc<<<blocks, kRegBlock, smem, h->stream>>>(x, mu, sigma, (const float4*)q.qpad, lq4, q.M,
                                                   Nw, out);
        CDTW_LAUNCH(h, "cdtw_regc_kernel");
        return CDTW_OK;
    }
    RegKernel k = per == 4   ? (euclid ? reg_kernels().eu4[q.W] : reg_kernels().mh4[q.W])
                  : per == 2 ? (euclid ? reg_kernels().eu2[q.W] : reg_kernels().mh2[q.W])
                             : (euclid ? reg_kernels().eu[q.W] : reg_kernels().mh[q.W]);
    if (smem > 48 * 1024)
        CDTW_CUDA(h, cudaFuncSetAttribute((const void*)k,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
    const unsigned blocks = (unsigned)div_up(div_up(L, per), kRegBlock);
    k<<<blocks, kRegBlock, smem, h->stream>>>(x, mu, sigma, (const float4*)q.qpad, lq4, q.M, Nw,
                                              idx, (int)L, out);
    CDTW_LAUNCH(h, "cdtw_reg_kernel");
    return CDTW_OK;
}

}  // namespace cdtw
