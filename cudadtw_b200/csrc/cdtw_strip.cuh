// Device code of the strip kernels (shared by the single- and multi-query
// searches).  Banded DTW for wide bands ("strip" kernel): one thread per window, the
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
#pragma once

#include "common.cuh"

#include <algorithm>

namespace cdtw {

// Per-query arguments of the strip kernels.
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

namespace {

constexpr int kStripWarps = 2;  // warps per block



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

__device__ __forceinline__ float qext(const StripArgs& a, int c) {
    return __ldg(a.qrev0 + (a.qbase - c));
}

template <int R>
__device__ __forceinline__ void load_q(const StripArgs& a, int c, float (&qv)[R]) {
    if constexpr (R >= 4) {
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
    } else {
#pragma unroll
        for (int r = 0; r < R; ++r) qv[r] = qext(a, c - r);
    }
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

// Resets a lane's ring to the virtual row -1 (D[-1][-1] = 0, +inf elsewhere).
__device__ __forceinline__ void ring_reset(float* ring, int P) {
    for (int s = 0; s < P; ++s) ring[s * 32] = CDTW_INF;
    ring[(P - 1) * 32] = 0.0f;  // column -1
}

// One strip (data rows j0..j0+R-1) of the window at xw: reads the previous
// strip's last row from the ring, writes this strip's last row to it.
// SEARCH: adds the strip rows' forward LB_Keogh terms to pre and returns the
// minimum of the strip's last row in rmin.  Control flow depends only on
// (M, W, R), so lanes of a warp may be at different windows and strips.
template <int R, bool EU, bool SEARCH>
__device__ __forceinline__ void strip_pass(const StripArgs& a, const float* __restrict__ xw,
                                           const Norm& nm, int j0, float* ring,
                                           const float2* __restrict__ qenv, float& pre,
                                           float& rmin) {
    const int M = a.M, W = a.W, P = a.P;
    const int n_int = 2 * W - 2 * R + 3;  // interior steps t = 2R-2 .. 2W (W >= R-1)
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
    rmin = CDTW_INF;
    // interior t = 2R-2 .. 2W: peel to a column that is a multiple of R ...
    int c = c0 + 2 * R - 2, it = 0;
    for (; it < n_int && (c & (R - 1)) != 0; ++it, ++c)
        interior_ldg<R, EU>(a, c, z, d1, d2, ring, rs, ws, dg0, rmin);
    // ... then whole blocks of R steps with the query in a register ring
    if (it + R <= n_int) {
        constexpr int PF = R < 8 ? R : 8;
        float qr[R];  // qr[i mod R] = qext[i]
#pragma unroll
        for (int s1 = 1; s1 < R; ++s1) qr[s1] = qext(a, c - R + s1);
        for (; it + R <= n_int; it += R, c += R) {
            // rs is a multiple of R here (P and c are), so the block's R read
            // slots rs..rs+R-1 do not wrap
            float upv[PF];  // ring values of the next PF steps, loaded together
#pragma unroll
            for (int u = 0; u < R; ++u) {
                if (u % PF == 0) {
#pragma unroll
                    for (int v = 0; v < PF; ++v) upv[v] = ring[(rs + u + v) * 32];
                }
                qr[u] = qext(a, c + u);
                strip_step<R, 0, R - 1, -1, EU>(
                    z, d1, d2, [&](int r) { return qr[(u - r + R) % R]; }, upv[u % PF], dg0);
                dg0 = upv[u % PF];
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
}

// D[M-1][M-1] after the last strip: D[M'-1][M'-1] of the extended matrix,
// at column M'-1 of the ring.
template <int R>
__device__ __forceinline__ float strip_result(const StripArgs& a, const float* ring) {
    const int S = (a.M + R - 1) / R;
    return ring[(((S * R - 1) % a.P)) * 32];
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
    ring_reset(ring, a.P);
    const int S = (a.M + R - 1) / R;
    float pre = 0.f, rmin;
    for (int s = 0; s < S; ++s) {
        strip_pass<R, EU, SEARCH>(a, xw, nm, s * R, ring, qenv, pre, rmin);
        if (SEARCH && s * R + R < a.M) {  // the strip's last row is a real row before M-1
            const float bsf = load_bsf(key);
            alive = alive && (rmin + lb_suffix(lbk, pre, a.M) * kLbSlack < bsf);
            if (!__any_sync(0xffffffffu, alive)) return CDTW_INF;
        }
    }
    return strip_result<R>(a, ring);
}

}  // namespace

}  // namespace cdtw
