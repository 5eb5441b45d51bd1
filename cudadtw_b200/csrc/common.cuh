// Internal definitions shared by the sm_100a kernels and the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdarg.h>
#include <math.h>
#include <string.h>

#include <vector>

#include "../../include/cudadtw.h"

#define CDTW_INF __int_as_float(0x7f800000)

namespace cdtw {

// ---- per-handle state ------------------------------------------------------

// Device layout of the prepared query ("query pack").  The reference keeps the
// z-normalised query and its envelope in __constant__ arrays
// (include/cdtw.cuh:9-11); here they live in one handle-owned device block:
//   qpad  : 4 shifted copies of the +inf-padded query, copy m holds
//           qp[a+m] where qp[a] = zq[a-W] (zq outside [0,M) = +inf).  Row j of
//           the register-band kernel reads qp[j..j+2W] with 16-byte loads from
//           copy (j&3) at index (j&~3).
//   env   : (L_k, U_k) pairs of the query envelope over +-W.
//   zq    : z-normalised query (float).
//   qrev  : 4 shifted copies of the reversed, extended query read by the strip
//           kernel: copy m holds qr[a+m], qr[b] = qext[qrev_base - b], with
//           qext[i] = +inf (i < 0), zq[i] (0 <= i < M), i*1e18 (i >= M).
//           Optional (nullptr: not built).
struct QueryPack {
    int M = 0, W = 0;
    int lq = 0;            // floats per qpad copy (multiple of 4)
    float* qpad = nullptr; // 4 * lq floats
    float2* env = nullptr; // M pairs
    float* zq = nullptr;   // M floats
    double* zq64 = nullptr;// M doubles
    int lqr = 0;           // floats per qrev copy (multiple of 4)
    int qrev_base = 0;     // A
    float* qrev = nullptr; // 4 * lqr floats
    float* qraw = nullptr; // M floats: the query as given (optional)
};

// Extent of the reversed extended query for strips of up to kStripRowsMax rows.
constexpr int kStripRowsMax = 32;
__host__ __device__ inline int qrev_lo(int W) { return -(W + kStripRowsMax + 8); }
__host__ __device__ inline int qrev_hi(int M, int W) { return M + W + 3 * kStripRowsMax + 8; }
__host__ __device__ inline int qrev_len(int M, int W) {
    return (qrev_hi(M, W) - qrev_lo(W) + 1 + 4 + 3) / 4 * 4;
}

}  // namespace cdtw

struct cdtw_handle_s {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    // grow-only device workspace
    void* ws = nullptr;
    size_t ws_bytes = 0;
    // cached plan of the batched search (batch_host.cu)
    void* batch = nullptr;
    // state of an incremental search over a stream (stream.cu)
    void* stream_state = nullptr;
    // cached plan of the batched search through concurrent pipelines (batch_pipe.cu)
    void* batch_pipe = nullptr;
    // boundary rings of the strip kernel's resident warps (grow-only)
    void* ring = nullptr;
    size_t ring_bytes = 0;
    // query pack storage (grow-only)
    void* qmem = nullptr;
    size_t qmem_bytes = 0;
    cdtw::QueryPack q;
    bool has_query = false;
    // cap on the device memory the handle holds (0: none), cdtw_set_memory_limit
    size_t mem_limit = 0;
    size_t batch_bytes = 0;  // device memory of the cached batched-search plan
    size_t stream_bytes = 0;  // device memory kept by the streaming search
    // small pinned host buffer for scalar results
    void* pinned = nullptr;
    // stage counts of the last search: windows, after LB_Kim, after LB_Keogh
    int64_t last_counts[4] = {0, 0, 0, 0};
    // the last search's best distance lies below the largest LB_Kim
    int last_flag = 0;
    // the last cdtw_pair_fwd with a path record recomputed from checkpoints
    int last_pair_recompute = 0;
    // cDTW kernel variant per band (0 = built-in rule); set by the autotuner
    unsigned char band_variant[CDTW_MAX_QUERY] = {0};
    // host-buffer pipeline (cdtw_all_windows_host): copy-in, copy-out and a
    // second compute stream, and an event pool, created on first use
    cudaStream_t xfer[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t xev[3 * 16 + 1] = {};
    bool xready = false;
    char err[512] = {0};
};

namespace cdtw {

int set_error(cdtw_handle h, int status, const char* fmt, ...);
// Bytes of a query pack for (M, W); with q and base, points q's arrays into
// base (device memory of at least that many bytes).
size_t query_pack_layout(int M, int W, QueryPack* q, char* base);
void batch_plan_release(cdtw_handle h);
void stream_release(cdtw_handle h);
void batch_pipe_release(cdtw_handle h);
int search_batched_pipelines(cdtw_handle h, const float* d_subject, int64_t N,
                             const float* h_queries, const std::vector<int>& M,
                             const std::vector<int>& W, int metric, int64_t* locations,
                             float* distances);
// top-k non-overlapping matches (search.cu)
size_t topk_workspace_bytes(int64_t N, int M, int W);
int run_topk(cdtw_handle h, const float* x, int64_t N, const double* mu, const float* sigma,
             bool euclid, int k, char* ws_base, std::vector<unsigned long long>* picks);
// the same with every step on the device (graph-capturable); k2 >= k picks
size_t topk_device_workspace_bytes(int64_t N, int M, int W, int k2);
int run_topk_device(cdtw_handle h, const float* x, int64_t N, const double* mu,
                    const float* sigma, bool euclid, int k, int k2, char* ws_base,
                    const int32_t* prev, const int* prev_n, int32_t* picks, float* pick_d,
                    int* npicks, int* status);
// topk_device.cu
int launch_topk_threshold(cdtw_handle h, const float* sd, int nseg, const float* prev_d,
                          const int* prev_n, int k2, unsigned long long* key, float* t_out);
int launch_topk_greedy(cdtw_handle h, const unsigned long long* hits, const int* nh, int cap,
                       int k2, int M, int* acc, int32_t* picks, float* pick_d, int* npicks,
                       int* status);
// pairwise cDTW forward / backward (pair.cu)
void pair_shape(int L, int W, int* G, int* C);
size_t pair_dirs_words(int L, int W);
int launch_pair_znorm(cdtw_handle h, const float* q, const float* s, int64_t n, int L, float* zq,
                      float* zs, double* hdr);
// qstride: elements between the queries of consecutive pairs (-1: L; 0: all
// pairs share the query at zq).  gate: a device count of the pairs present
// (the first min(n, *gate) run; warps past them exit at once), and the
// launch does nothing when *gate > gate_max (decisions the host cannot see).
// gate_min: the launch also does nothing when *gate <= gate_min; wide: (no
// path record) lane groups of 32 with the fewest cells per lane -- the
// shortest step, for a handful of pairs.
int launch_pair_fwd(cdtw_handle h, const float* zq, const float* zs, int64_t n, int L, int W,
                    bool euclid, float* D, uint32_t* dirs, uint32_t* rows, uint32_t* cols,
                    int64_t qstride = -1, const int* gate = nullptr, int gate_max = 0,
                    int gate_min = -1, bool wide = false);
// Checkpointed path record (memory: pair_ckpt_floats per pair instead of the
// direction scratch); pair_ckpt_floats is 0 where the mode does not apply.
size_t pair_ckpt_floats(int L, int W);
int launch_pair_fwd_ckpt(cdtw_handle h, const float* zq, const float* zs, int64_t n, int L,
                         int W, bool euclid, float* D, float* ckpt, uint32_t* rows,
                         uint32_t* cols);
int launch_pair_bwd(cdtw_handle h, const float* q, const float* s, int64_t n, int L,
                    const double* hdr, const uint32_t* rows, const uint32_t* cols,
                    const float* dD, bool euclid, float* dq, float* ds);
int check_cuda(cdtw_handle h, cudaError_t e, const char* what);
int ensure_workspace(cdtw_handle h, size_t bytes);
// CDTW_ENOMEM when the handle would hold more than its memory limit after
// releasing `freed` bytes and allocating `bytes` more.
int check_memory_limit(cdtw_handle h, size_t freed, size_t bytes, const char* what);

#define CDTW_TRY(expr)                        \
    do {                                      \
        int _st = (expr);                     \
        if (_st != CDTW_OK) return _st;       \
    } while (0)

#define CDTW_CUDA(h, call) CDTW_TRY(::cdtw::check_cuda((h), (call), #call))
#define CDTW_LAUNCH(h, what) CDTW_TRY(::cdtw::check_cuda((h), cudaGetLastError(), (what)))

__host__ __device__ inline int64_t div_up(int64_t a, int64_t b) { return (a + b - 1) / b; }
__host__ __device__ inline int64_t round_up(int64_t a, int64_t b) { return div_up(a, b) * b; }

// Three-input minimum (PTX ISA 8.8, sm_100+): one instruction for the three
// DTW predecessors.  NaN-ignoring like fminf.
__device__ __forceinline__ float min3f(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float max3f(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// Cell cost of the reference kernels: (z-q)^2 or |z-q| (cdtw.cuh:235-240).
template <bool EUCLID>
__device__ __forceinline__ float cell(float d, float m) {
    return EUCLID ? fmaf(d, d, m) : fabsf(d) + m;
}

// Per-window normalisation constants from FP64 mean / FP32 sigma:
// z = (x - mu_hi) * s + c with mu = mu_hi + mu_lo (double-float) and
// c = -mu_lo * s.  x - mu_hi is exact up to one rounding of the (small)
// difference, so level-shifted windows keep full FP32 precision in z.
struct Norm {
    float mhi, s, c;
};
__device__ __forceinline__ Norm make_norm(double mu, float sigma) {
    Norm n;
    n.mhi = (float)mu;
    const float mlo = (float)(mu - (double)n.mhi);
    n.s = 1.0f / sigma;
    n.c = -mlo * n.s;
    return n;
}
__device__ __forceinline__ float znorm(const Norm& n, float x) {
    return fmaf(x - n.mhi, n.s, n.c);
}

// LB_Kim of the reference GPU path on ten z-normalised window samples
// s[0..4] (front) / s[5..9] (back) and the matching query values q[0..9]:
// 5x5 unconstrained DTW at the front (min over its last row and column) plus
// the 5x5 back block entered anywhere on its first row/column, the
// recurrences of include/bounds.cuh:315-404.  The two parts are independent:
// lb_kim_front + lb_kim_back, added in that order, is the bound.  (Seeding
// the search from the front part alone, the back part computed only where
// the front part passes, was measured: its seeds are poor enough that the
// first best-so-far prunes almost nothing on some queries.)
template <bool EU>
__device__ __forceinline__ float lb_kim_front(const float* s, const float* q) {
    auto lp = [](float d) { return EU ? d * d : fabsf(d); };
    float F[5], G[5];
    F[0] = lp(q[0] - s[0]);
#pragma unroll
    for (int k = 1; k < 5; ++k) F[k] = lp(q[0] - s[k]) + F[k - 1];
    float mem = F[4];
#pragma unroll
    for (int r = 1; r < 5; ++r) {
        G[0] = lp(q[r] - s[0]) + F[0];
#pragma unroll
        for (int k = 1; k < 5; ++k) G[k] = lp(q[r] - s[k]) + min3f(G[k - 1], F[k - 1], F[k]);
        mem = fminf(mem, G[4]);
#pragma unroll
        for (int k = 0; k < 5; ++k) F[k] = G[k];
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) mem = fminf(mem, F[k]);
    return mem;
}

// s / q: the last five window samples / query values.
template <bool EU>
__device__ __forceinline__ float lb_kim_back(const float* s, const float* q) {
    auto lp = [](float d) { return EU ? d * d : fabsf(d); };
    float F[5], G[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) F[k] = lp(q[0] - s[k]);
#pragma unroll
    for (int r = 1; r < 5; ++r) {
        G[0] = lp(q[r] - s[0]);
#pragma unroll
        for (int k = 1; k < 5; ++k) G[k] = lp(q[r] - s[k]) + min3f(G[k - 1], F[k - 1], F[k]);
#pragma unroll
        for (int k = 0; k < 5; ++k) F[k] = G[k];
    }
    return F[4];
}

template <bool EU>
__device__ __forceinline__ float lb_kim_dp(const float (&s)[10], const float (&q)[10]) {
    return lb_kim_front<EU>(s, q) + lb_kim_back<EU>(s + 5, q + 5);
}

// Packed (distance, index) key for the fused argmin: distances are >= 0 so
// their float bits order like unsigned ints; ties keep the lowest index
// (UCR's first strict minimum, UCR_DTW_BIN.cpp:682).
__host__ __device__ inline unsigned long long pack_key(float d, uint32_t idx) {
#ifdef __CUDA_ARCH__
    return ((unsigned long long)__float_as_uint(d) << 32) | idx;
#else
    uint32_t b;
    memcpy(&b, &d, 4);
    return ((unsigned long long)b << 32) | idx;
#endif
}

// Smallest packed (distance, index) key over the lanes of a warp: the least
// distance bits, then the lowest index among the lanes holding them; equal to
// the minimum of pack_key over the lanes with ok set (distances >= 0), ~0 when
// no lane has it.  All 32 lanes call.
__device__ __forceinline__ unsigned long long warp_min_key(bool ok, float d, uint32_t idx) {
    const unsigned db = ok ? __float_as_uint(d) : 0xffffffffu;
    const unsigned dmin = __reduce_min_sync(0xffffffffu, db);
    const unsigned im = __reduce_min_sync(0xffffffffu, (ok && db == dmin) ? idx : 0xffffffffu);
    return ((unsigned long long)dmin << 32) | im;
}

// A search candidate: window, its best lower bound, and its forward LB_Keogh
// (the sum whose suffixes give the cumulative bound for early abandoning).
struct Cand {
    int w;
    float lb;
    float lbk;
};

// Number of seed windows whose cDTW gives a query its first best-so-far:
// about kSeedCells band cells in total (a few tens of microseconds of cDTW),
// at least 64 and at most 4096 windows.
constexpr double kSeedCells = 2.0e8;
__host__ __device__ inline int seed_target(int M, int W) {
    const double cells = (double)M * (2.0 * W + 1.0) - (double)W * (W + 1.0);
    const double n = kSeedCells / (cells > 1.0 ? cells : 1.0);
    return n < 64.0 ? 64 : (n > 4096.0 ? 4096 : (int)n);
}

// Lower bounds are compared against the best-so-far with this relative
// slack, so FP32 rounding of a bound can never prune a window whose distance
// is below the best (a bound prunes only if it exceeds bsf by 1e-4).
constexpr float kLbSlack = 1.0f - 1e-4f;

// The forward LB_Keogh of the rows after a prefix, as a certain lower bound:
// lbk (all M rows) and pre (the prefix) are FP32 sums of non-negative terms,
// each within (M-1) * 2^-24 relative of its exact value whatever the order of
// summation (the filter kernels and the cDTW kernels sum in different orders
// and with or without fused multiply-adds), so lbk (1 - e) - pre (1 + e) with
// e = M * 1.2e-7 never exceeds the exact remainder.
__device__ __forceinline__ float lb_suffix(float lbk, float pre, int M) {
    const float e = (float)M * 1.2e-7f;
    return fmaxf(fmaf(lbk, 1.f - e, -pre * (1.f + e)), 0.f);
}

__device__ __forceinline__ float key_dist(unsigned long long k) {
    return __uint_as_float((unsigned)(k >> 32));
}
__device__ __forceinline__ float load_bsf(const unsigned long long* key) {
    const unsigned long long k = *(const volatile unsigned long long*)key;
    const float d = key_dist(k);
    return (k == ~0ull) ? CDTW_INF : d;
}

// Where a search kernel puts a finished window: without a hit list, the
// packed (distance, window) atomicMin into *key (argmin search); with one,
// every window whose packed key is below *key is appended to the list (the
// key then holds a fixed threshold that also drives the early abandoning:
// top-k candidate collection).  Appends past cap are counted, not stored.
struct HitSink {
    unsigned long long* hits = nullptr;
    int* n = nullptr;
    int cap = 0;
};

__device__ __forceinline__ void report_window(unsigned long long* key, const HitSink& s,
                                              float res, uint32_t w) {
    const unsigned long long k = pack_key(res, w);
    if (!s.hits) {
        atomicMin(key, k);
        return;
    }
    if (k < *(const volatile unsigned long long*)key) {
        const int at = atomicAdd(s.n, 1);
        if (at < s.cap) s.hits[at] = k;
    }
}

// ---- kernel launchers (defined in the .cu files) ----------------------------

int launch_avg_std(cdtw_handle h, const float* x, int64_t N, int M, double* mu, float* sigma);
int launch_avg_std64(cdtw_handle h, const float* x, int64_t N, int M, double* mu, double* sigma);
int launch_avg_std64(cdtw_handle h, const double* x, int64_t N, int M, double* mu, double* sigma);
// Exact FP64 argmin (lowest index on ties) of d[0..n): block partials then one
// final block; the result (value, index) lands in *res.
struct ArgMin64 {
    double v;
    long long i;
};
int launch_argmin64(cdtw_handle h, const double* d, int64_t n, ArgMin64* partial,
                    ArgMin64* res);
size_t argmin64_partials(int64_t n);
int launch_znorm64(cdtw_handle h, const double* q, int M, double* zq);
int launch_ed(cdtw_handle h, const double* x, int64_t N, const double* zq, int M,
              const double* sigma, double* out);
int launch_ldtw(cdtw_handle h, const float* x, int64_t N, const double* mu, const double* sigma,
                bool euclid, double* out);
// The reference's FP32 LDTW (ztsh2_ldtw / tsh2_ldtw arithmetic); qwork: M
// floats of device scratch for the reference-normalised query.
int launch_ldtw_ref(cdtw_handle h, const float* x, int64_t N, bool euclid, bool znorm,
                    float* qwork, float* out);
// Packed (float bits, index) minimum of out[0..n) into *key (first strict
// minimum; NaN skipped); *key must start at ~0.
int launch_argmin_f32(cdtw_handle h, const float* v, int64_t n, unsigned long long* key);
int launch_prepare_query(cdtw_handle h, const float* d_query_raw, int M, int W);
// One block per query: prepares packs[q] from the raw query at raw + offs[q].
int launch_prepare_queries(cdtw_handle h, const float* raw, const int64_t* offs,
                           const QueryPack* packs, int nq, int max_m);
int launch_cdtw_windows(cdtw_handle h, const float* x, int64_t N, const double* mu,
                        const float* sigma, const int32_t* idx, int64_t L, bool euclid,
                        float* out);
int launch_cdtw_strip(cdtw_handle h, const float* x, int64_t N, const double* mu,
                      const float* sigma, const int32_t* idx, int64_t L, bool euclid, int R,
                      float* out);
int strip_rows_default(int W);
// Lane-block kernels (cdtw_lane.cu): band spread over G lanes of B cells.
bool lane_shape(int W, int* G, int* B);
int lane_qpad_min(int M, int W);  // floats per query copy they read
int launch_cdtw_lane(cdtw_handle h, const float* x, int64_t N, const double* mu,
                     const float* sigma, const int32_t* idx, int64_t L, bool euclid, float* out);
int launch_cdtw_lane_search(cdtw_handle h, const float* x, int64_t N, const double* mu,
                            const float* sigma, const Cand* cands, const int* count, int* work,
                            int max_count, bool euclid, unsigned long long* key,
                            const HitSink& sink);
// floats per shifted query copy (QueryPack::lq) of a handle's query pack
inline int qpad_len(int M, int W) { return (int)(((int64_t)M + 2 * W + 56 + 3) / 4 * 4); }
// Kernel choice for band W: CDTW_VARIANT_REGISTER (one thread per window, band
// in registers, W <= 96), CDTW_VARIANT_STRIP16 / STRIP32 (strips of 16 / 32
// rows, W >= 15 / 31), CDTW_VARIANT_LANE (band over a lane group, 27 <= W <=
// 767).
int choose_variant(cdtw_handle h, int W);
int max_register_band();
int launch_lb_kim(cdtw_handle h, const float* x, int64_t N, const double* mu, const float* sigma,
                  const int32_t* idx, int64_t L, bool euclid, float* out,
                  unsigned long long* seeds = nullptr, unsigned* bmax = nullptr);
// The search's first pass: LB_Kim of every window into out (256-byte
// aligned), per 256 windows the smallest (seeds) and the largest (bmax).
int launch_lb_kim_all(cdtw_handle h, const float* x, int64_t N, const double* mu,
                      const float* sigma, bool euclid, float* out, unsigned long long* seeds,
                      unsigned* bmax);
size_t stream_envelope_scratch_bytes(int64_t N);
// gate: when set, the kernel does nothing if *gate <= gate_max (a device
// count the host cannot see, e.g. the LB_Kim survivors of a search).
int launch_stream_envelope(cdtw_handle h, const float* x, int64_t N, int W, float* scratch,
                           float2* env, const int* gate = nullptr, int gate_max = 0);
int launch_lb_keogh(cdtw_handle h, const float* x, int64_t N, const double* mu,
                    const float* sigma, const float2* xenv, const int32_t* idx, int64_t L,
                    bool euclid, float* fwd, float* rev);
// DTW over a device candidate list with early abandoning and a fused argmin
// into *key (packed distance/index), or, with a hit list, the collection of
// the windows below the threshold in *key.  `count` and `work` are device
// ints.
int launch_cdtw_search(cdtw_handle h, const float* x, int64_t N, const double* mu,
                       const float* sigma, const Cand* cands, const int* count, int* work,
                       int max_count, bool euclid, unsigned long long* key,
                       const HitSink& sink = HitSink());
// init_key: a device key the search starts from (a bound carried over from
// earlier parts of a stream), else no bound.
int run_search(cdtw_handle h, const float* x, int64_t N, const double* mu, const float* sigma,
               bool euclid, char* ws_base, unsigned long long** key_out, int** ctr_out,
               const unsigned long long* init_key = nullptr);
size_t search_workspace_bytes(int64_t N, int M, int W);

}  // namespace cdtw
