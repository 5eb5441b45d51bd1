// Banded DTW for wide bands ("strip" kernel): one thread per window, the
// window processed in strips of R data rows by persistent warps.
//
// Reference: the block kernels of include/cdtw.cuh:164-363 refuse bands whose
// W+2 lanes or 3(W+2)+M shared words do not fit (cdtw.cuh:459-465).  Here a
// thread keeps R rows of the band in registers and walks them along
// anti-diagonals: at step t, row r of the strip updates query column
// c_t - r, so the R cells of a step are independent (no left-to-right chain)
// and each depends only on the previous two steps.  The values a strip
// hands to the next one (its last row, one per query column) go through a
// per-lane ring of P >= 2W+2 floats.  The ring lives in global memory, one
// slice per resident warp (slot-major, so a warp's 32 lanes touch one
// 128-byte line per access), small enough in total to stay in L2; occupancy
// is then set by registers, not by shared memory.  The query values of a
// step are the same for all 32 lanes: in the aligned body of a strip they sit
// in a register ring indexed by column mod R (one scalar load per step); the
// other steps read them with broadcast 16-byte loads from four shifted copies
// of the reversed query.
//
// Band edges: row r of a strip is inside the band for steps [2r, 2W+2r]; the
// entry and exit triangles of a strip are unrolled at compile time, so there
// is no per-cell masking.  Matrix edges: query columns < 0 are +inf; data
// rows and query columns >= M are extended to the next multiple of R with
// "diagonal-only" cells: e_k = k * 1e18 at position k, so cost(k,k) = 0 and
// every other extended cell costs >= 1e36 (or +inf).  D[M'-1][M'-1] of the
// extended matrix therefore equals D[M-1][M-1] exactly, and it is the last
// row of the last strip, read back from the ring.
#include "common.cuh"

#include <algorithm>

namespace cdtw {

namespace {

constexpr int kStripWarps = 2;  // warps per block

struct StripArgs {
    const float* x;
    const double* mu;
    const float* sigma;
    const float4* qrev4;  // 4 copies of the reversed extended query, lqr floats each
    const float* qrev0;   // copy 0: qext[i] = qrev0[qbase - i]
    int lqr4;             // float4 per copy
    int qbase;            // A
    int M, W, P, Nw;      // P: ring slots per lane, a multiple of R, >= 2W+2
    float* ring;          // rings of all resident warps, P*32 floats each
    const int32_t* idx;
    int L;
    float* out;
};

__device__ __forceinline__ float ext_value(int k) { return (float)k * 1e18f; }

// One anti-diagonal step over rows [LO, HI] of the strip.
//   z[r]    : z-normalised sample of row r (static for the strip)
//   d1[r]   : row r at step t-1 (becomes row r at step t)
//   d2[r]   : row r at step t-2 (becomes row r at step t-1)
//   q(r)    : query value at column c_t - r
//   up0/dg0 : previous-strip values at columns c_t and c_t - 1 (row 0 only)
template <int R, int LO, int HI, int KILL, bool EU, class QF>
__device__ __forceinline__ void strip_step(const float (&z)[R], float (&d1)[R], float (&d2)[R],
                                           QF q, float up0, float dg0) {
#pragma unroll
    for (int r = HI; r >= LO; --r) {  // bottom-up: row r-1 still holds step t-1 / t-2
        const float up = (r == 0) ? up0 : d1[r - 1];
        const float dg = (r == 0) ? dg0 : d2[r - 1];
        const float v = cell<EU>(z[r] - q(r), min3f(dg, up, d1[r]));
        d2[r] = d1[r];
        d1[r] = v;
    }
    if (KILL >= 0) {  // row KILL just left the band: it must read as +inf below
        d2[KILL] = d1[KILL];
        d1[KILL] = CDTW_INF;
    }
}

template <int R>
__device__ __forceinline__ void load_q(const StripArgs& a, int c, float (&qv)[R]) {
    const int a0 = a.qbase - c;  // qrev index of row 0's query value
    const float4* p = a.qrev4 + (a0 & 3) * a.lqr4 + (a0 >> 2);
#pragma unroll
    for (int k = 0; k < R / 4; ++k) {
        const float4 v = __ldg(p + k);
        qv[4 * k + 0] = v.x;
        qv[4 * k + 1] = v.y;
        qv[4 * k + 2] = v.z;
        qv[4 * k + 3] = v.w;
    }
}

__device__ __forceinline__ float qext(const StripArgs& a, int c) {
    return __ldg(a.qrev0 + (a.qbase - c));
}

__device__ __forceinline__ int wrap_inc(int s, int P) { return (s + 1 == P) ? 0 : s + 1; }

// Compile-time loop over the entry triangle: steps t = T .. 2R-3.
template <int R, int T, bool EU>
struct Entry {
    __device__ __forceinline__ static void run(const StripArgs& a, int c0, const float (&z)[R],
                                               float (&d1)[R], float (&d2)[R], float* ring,
                                               int& rs, float& dg0) {
        if constexpr (T <= 2 * R - 3) {
            float qv[R];
            load_q<R>(a, c0 + T, qv);
            const float up0 = ring[rs * 32];
            strip_step<R, 0, T / 2, -1, EU>(z, d1, d2, [&](int r) { return qv[r]; }, up0, dg0);
            dg0 = up0;
            rs = wrap_inc(rs, a.P);
            Entry<R, T + 1, EU>::run(a, c0, z, d1, d2, ring, rs, dg0);
        }
    }
};

// Compile-time loop over the exit triangle: steps t = 2W+1+TP, TP = 0 .. 2R-3.
template <int R, int TP, bool EU>
struct Exit {
    __device__ __forceinline__ static void run(const StripArgs& a, int cx, const float (&z)[R],
                                               float (&d1)[R], float (&d2)[R], float* ring,
                                               int& ws, float& rmin) {
        if constexpr (TP <= 2 * R - 3) {
            float qv[R];
            load_q<R>(a, cx + TP, qv);
            constexpr int LO = (TP + 2) / 2;  // rows r with 2r >= TP+1
            constexpr int KILL = (TP % 2 == 0) ? TP / 2 : -1;
            strip_step<R, LO, R - 1, KILL, EU>(z, d1, d2, [&](int r) { return qv[r]; }, 0.f, 0.f);
            ring[ws * 32] = d1[R - 1];
            rmin = fminf(rmin, d1[R - 1]);
            ws = wrap_inc(ws, a.P);
            Exit<R, TP + 1, EU>::run(a, cx, z, d1, d2, ring, ws, rmin);
        }
    }
};

// Interior step with the query values read from memory (peel / remainder).
template <int R, bool EU>
__device__ __forceinline__ void interior_ldg(const StripArgs& a, int c, const float (&z)[R],
                                             float (&d1)[R], float (&d2)[R], float* ring,
                                             int& rs, int& ws, float& dg0, float& rmin) {
    float qv[R];
    load_q<R>(a, c, qv);
    const float up0 = ring[rs * 32];
    strip_step<R, 0, R - 1, -1, EU>(z, d1, d2, [&](int r) { return qv[r]; }, up0, dg0);
    dg0 = up0;
    rs = wrap_inc(rs, a.P);
    ring[ws * 32] = d1[R - 1];
    rmin = fminf(rmin, d1[R - 1]);
    ws = wrap_inc(ws, a.P);
}

// DTW of window w through the strips.  SEARCH: abandon (return +inf) once the
// last row of a strip plus the remaining forward LB_Keogh suffix reaches the
// best-so-far for every lane of the warp; all 32 lanes must call together.
template <int R, bool EU, bool SEARCH>
__device__ __forceinline__ float strip_dtw(const StripArgs& a, int w, float* ring,
                                           const float2* __restrict__ qenv, float lbk,
                                           bool& alive, const unsigned long long* key) {
    const Norm nm = make_norm(a.mu[w], a.sigma[w]);
    const float* __restrict__ xw = a.x + w;
    const int M = a.M, W = a.W, P = a.P;
    // ring: previous-strip row values by query column, slot = col mod P;
    // virtual row -1: D[-1][-1] = 0, +inf elsewhere
    for (int s = 0; s < P; ++s) ring[s * 32] = CDTW_INF;
    ring[(P - 1) * 32] = 0.0f;  // column -1
    const int S = (M + R - 1) / R;
    const int n_int = 2 * W - 2 * R + 3;  // interior steps t = 2R-2 .. 2W (W >= R-1)
    float pre = 0.f;
    for (int s = 0; s < S; ++s) {
        const int j0 = s * R;
        float z[R], d1[R], d2[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int j = j0 + r;
            z[r] = (j < M) ? znorm(nm, __ldg(xw + j)) : ext_value(j);
            d1[r] = CDTW_INF;
            d2[r] = CDTW_INF;
            if (SEARCH && j < M) {
                const float2 e = __ldg(qenv + j);
                const float dl = max3f(z[r] - e.y, e.x - z[r], 0.f);
                pre += EU ? dl * dl : dl;
            }
        }
        const int c0 = j0 - W;  // row 0's column at step 0
        int rs = ((c0 % P) + P) % P;                      // read slot: column c_t
        int ws = (((c0 - (R - 1)) % P) + P) % P;          // write slot: column c_t - (R-1)
        float dg0 = ring[(rs == 0 ? P - 1 : rs - 1) * 32];  // column c0 - 1
        // entry triangle: t = 0 .. 2R-3 (no writes yet: row R-1 starts at 2R-2)
        Entry<R, 0, EU>::run(a, c0, z, d1, d2, ring, rs, dg0);
        ws = (ws + 2 * R - 2) % P;  // column c_t - (R-1) for the first write at t = 2R-2
        float rmin = CDTW_INF;      // minimum of the strip's last row (search only)
        // interior t = 2R-2 .. 2W: peel to a column that is a multiple of R ...
        int c = c0 + 2 * R - 2, it = 0;
        for (; it < n_int && (c & (R - 1)) != 0; ++it, ++c)
            interior_ldg<R, EU>(a, c, z, d1, d2, ring, rs, ws, dg0, rmin);
        // ... then whole blocks of R steps with the query in a register ring
        if (it + R <= n_int) {
            float qr[R];  // qr[i mod R] = qext[i]
#pragma unroll
            for (int s1 = 1; s1 < R; ++s1) qr[s1] = qext(a, c - R + s1);
            for (; it + R <= n_int; it += R, c += R) {
                // rs is a multiple of R here (P and c are), so the block's R
                // read slots rs..rs+R-1 do not wrap
                float upv[8];  // ring values of the next 8 steps, loaded together
#pragma unroll
                for (int u = 0; u < R; ++u) {
                    if (u % 8 == 0) {
#pragma unroll
                        for (int v = 0; v < 8; ++v) upv[v] = ring[(rs + u + v) * 32];
                    }
                    qr[u] = qext(a, c + u);
                    strip_step<R, 0, R - 1, -1, EU>(
                        z, d1, d2, [&](int r) { return qr[(u - r + R) % R]; }, upv[u % 8], dg0);
                    dg0 = upv[u % 8];
                    ring[ws * 32] = d1[R - 1];
                    if (SEARCH) rmin = fminf(rmin, d1[R - 1]);
                    ws = wrap_inc(ws, P);
                }
                rs += R;
                if (rs == P) rs = 0;
            }
        }
        // ... and the remaining steps
        for (; it < n_int; ++it, ++c) interior_ldg<R, EU>(a, c, z, d1, d2, ring, rs, ws, dg0, rmin);
        // exit triangle: t = 2W+1 .. 2W+2R-2 (row 0 done, no reads)
        Exit<R, 0, EU>::run(a, c0 + 2 * W + 1, z, d1, d2, ring, ws, rmin);
        ring[ws * 32] = CDTW_INF;  // column j0+R+W: outside the next strip's upper band edge
        if (SEARCH && j0 + R < M) {  // the strip's last row is a real row before M-1
            const float bsf = load_bsf(key);
            alive = alive && (rmin + (lbk - pre) * kLbSlack < bsf);
            if (!__any_sync(0xffffffffu, alive)) return CDTW_INF;
        }
    }
    // D[M'-1][M'-1] of the extended matrix = D[M-1][M-1]; it sits at column M'-1
    return ring[(((S * R - 1) % P)) * 32];
}

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
                         int* __restrict__ work, unsigned long long* __restrict__ key) {
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
        if (i < n && res < CDTW_INF) atomicMin(key, pack_key(res, (uint32_t)c.w));
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
                             int max_count, bool euclid, int R, unsigned long long* key) {
    const QueryPack& q = h->q;
    if (R != 16 && R != 32) return set_error(h, CDTW_EINVAL, "strip rows must be 16 or 32");
    if (q.W < R - 1)
        return set_error(h, CDTW_EUNSUPPORTED, "strip kernel needs W >= R-1 (W=%d R=%d)", q.W, R);
    if (max_count <= 0) return CDTW_OK;
    using SK = void (*)(const StripArgs, const float2*, const Cand*, const int*, int*,
                        unsigned long long*);
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
    k<<<blocks, kStripWarps * 32, 0, h->stream>>>(a, q.env, cands, count, work, key);
    CDTW_LAUNCH(h, "cdtw_strip_search_kernel");
    return CDTW_OK;
}

}  // namespace cdtw
