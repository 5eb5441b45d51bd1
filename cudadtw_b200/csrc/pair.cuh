// Differentiable pairwise cDTW, forward device code (no reference
// counterpart; the DP is the
// banded recurrence of include/cdtw.cuh:24-88 / UCR_DTW_BIN.cpp:288-354 on
// two series of equal length L).
//
// Forward: one group of G lanes (a power of two) per pair walks the band
// anti-diagonal by anti-diagonal.  Anti-diagonal k = i + j holds the band
// cells d = j - i with d = k (mod 2), |d| <= W; slot p = (d + W - e) / 2 with
// e = (k + W) & 1, so every anti-diagonal has W + 1 slots and lane l owns
// slots [l*C, l*C + C).  A cell needs slot p (diag) from k-2 and slots p, p-1
// (e = 0) or p+1, p (e = 1) from k-1: one shuffle per step.  The query values
// of a lane's cells move by one position every second step and the subject
// values every other step; the windows are rotated by index (the step loop
// is unrolled 2C times) and refilled by a shuffle from the neighbouring lane,
// the edge lanes reading the pair's series from global memory (L2-resident).
//
// With a path record the forward also stores 2 bits per band cell (diagonal
// predecessor is the minimum; up <= left) in device scratch, one element of
// 2C bits per lane and anti-diagonal (a byte for C <= 4, 16 bits for C <= 8,
// else 32), and, once the pair is done, one lane backtracks from (L-1, L-1)
// to (0, 0) and writes the warping path as row runs [a_i, b_i] and column
// runs [c_j, d_j].  Backward
// sums the cost derivatives over those runs and applies the z-normalisation
// Jacobian (I - 11'/L - zz'/L) / sigma.
#pragma once

#include "common.cuh"

#include <algorithm>
#include <type_traits>
#include <utility>

namespace cdtw {

constexpr int kPairThreads = 128;
constexpr int kWalkChunk = 64;  // bytes of direction record per lane in one backtracking chunk
constexpr unsigned kFull = 0xffffffffu;

struct PairArgs {
    const float* zq;      // DP inputs: n x L (z-normalised copies or the raw series);
    const float* zs;      // pair p's query starts at zq + p * qstride (0: one shared query)
    int64_t qstride;
    int64_t n;
    int L, W, G, lgG;
    float* D;             // n outputs
    uint32_t* dirs;       // per pair dstride words: 2L-1 rows of G lane elements (path record)
    int dstride;
    int recb, logb;       // shared-record mode: bytes of record and move log per group
    const int* gate;      // when set: a device count of the pairs present (at most n);
    int gate_max;         // the launch does nothing when it exceeds gate_max
    int gate_min;         // or when it is at most gate_min
    uint32_t* rows;       // per pair L words: a_i | b_i << 16
    uint32_t* cols;       // per pair L words: c_j | d_j << 16
    float* ckpt;          // checkpointed mode: per pair nseg x 2C x G floats
    int seg;              // anti-diagonals per segment (a multiple of 2C)
    int nseg;             // segments per pair
};

namespace {


// z-value of one sample with the pair header's mean and sigma (shared by the
// forward preparation and the backward pass, so both see the same floats).
__device__ __forceinline__ float pair_z(float x, double mu, double inv) {
    return (float)(((double)x - mu) * inv);
}

// Direction bits of one cell, as predicated ORs of immediates: bit SH when
// the diagonal is the minimum, bit SH+1 when up <= left.
template <int SH>
__device__ __forceinline__ void dir_bits(uint32_t& w, float diag, float m, float up, float left) {
    asm("{\n\t.reg .pred p;\n\tsetp.eq.f32 p, %1, %2;\n\t@p or.b32 %0, %0, %3;\n\t}"
        : "+r"(w) : "f"(diag), "f"(m), "n"(1u << SH));
    asm("{\n\t.reg .pred p;\n\tsetp.le.f32 p, %1, %2;\n\t@p or.b32 %0, %0, %3;\n\t}"
        : "+r"(w) : "f"(up), "f"(left), "n"(2u << SH));
}

// Direction element of one lane and anti-diagonal: 2 bits per slot.
template <int C>
using DirT = std::conditional_t<(C <= 4), uint8_t, std::conditional_t<(C <= 8), uint16_t, uint32_t>>;

// One cell (compile-time slot c) of an anti-diagonal of parity E.
template <int C, bool EU, bool DIRS, int E, int RQ, int RS, int c>
__device__ __forceinline__ void dp_cell(float (&X)[C], const float (&Y)[C], const float (&Q)[C],
                                        const float (&Sv)[C], const float (&lim)[C], float nb,
                                        uint32_t& nbits) {
    const float up = (E == 0) ? Y[c] : (c == C - 1 ? nb : Y[c + 1 < C ? c + 1 : c]);
    const float left = (E == 0) ? (c == 0 ? nb : Y[c > 0 ? c - 1 : 0]) : Y[c];
    const float diag = X[c];
    const float m = min3f(diag, up, left);
    const float df = __fsub_rn(Q[(c - RQ % C + C) % C], Sv[(c + RS) % C]);
    float v = EU ? __fmaf_rn(df, df, m) : __fadd_rn(fabsf(df), m);
    if (E == 1) v = fmaxf(v, lim[c]);  // d = W + 1 lies outside the band
    X[c] = v;
    if constexpr (DIRS) dir_bits<2 * c>(nbits, diag, m, up, left);
}

template <int C, bool EU, bool DIRS, int E, int RQ, int RS, int... Cs>
__device__ __forceinline__ void dp_cells_seq(float (&X)[C], const float (&Y)[C],
                                             const float (&Q)[C], const float (&Sv)[C],
                                             const float (&lim)[C], float nb, uint32_t& nbits,
                                             std::integer_sequence<int, Cs...>) {
    (dp_cell<C, EU, DIRS, E, RQ, RS, Cs>(X, Y, Q, Sv, lim, nb, nbits), ...);
}

// One anti-diagonal of parity E: X (slots of k-2) becomes k from Y (k-1).
// Logical query value of slot c is Q[(c - RQ) mod C], subject value
// Sv[(c + RS) mod C].
template <int C, bool EU, bool DIRS, int E, int RQ, int RS>
__device__ __forceinline__ void dp_cells(float (&X)[C], const float (&Y)[C], const float (&Q)[C],
                                         const float (&Sv)[C], const float (&lim)[C], float nb,
                                         uint32_t& bits) {
    uint32_t nbits = 0;
    dp_cells_seq<C, EU, DIRS, E, RQ, RS>(X, Y, Q, Sv, lim, nb, nbits,
                                         std::make_integer_sequence<int, C>{});
    if (DIRS) bits = nbits;
}

// State of one lane of a pair's group during the forward DP.
template <int C>
struct PairLane {
    float A[C], B[C], Q[C], Sv[C], lim[C];
    uint32_t bits;  // direction bits of the last anti-diagonal
    int iq, js;    // lane 0's slot-0 query index, lane G-1's last-slot subject index
    float pq, ps;  // the values at iq + 1 / js + 1 (the next shift's)
};

// Direction element of anti-diagonal k: to the pair's global record (DM 1,
// live groups only) or to the group's shared-memory record (DM 2).
template <int C, int DM>
__device__ __forceinline__ void store_dirs(const PairLane<C>& st, uint32_t* drow, int G, int l,
                                           int k, bool live) {
    if constexpr (DM == 1 || DM == 2) {
        if (DM == 2 || live) ((DirT<C>*)drow)[(size_t)k * G + l] = (DirT<C>)st.bits;
    }
}

// Step with parity 1 (subject window shifts first; post-shift rotation RS)
// writing B from A; step with parity 0 (query window shifts; rotation RQ)
// writing A from B.
template <int C, bool EU, bool DIRS, int RQ, int RS>
__device__ __forceinline__ void step_odd(PairLane<C>& st, const float* ss, int L, int G, int l,
                                         bool shift) {
    if (shift) {
        constexpr int slot = (RS - 1 + C) % C;
        const float v = __shfl_down_sync(kFull, st.Sv[slot], 1, G);
        st.Sv[slot] = (l == G - 1) ? st.ps : v;
        if (l == G - 1) {
            ++st.js;
            st.ps = st.js + 1 < L ? __ldg(ss + st.js + 1) : 0.f;
        }
    }
    float nb = __shfl_down_sync(kFull, st.A[0], 1, G);
    if (l == G - 1) nb = CDTW_INF;
    dp_cells<C, EU, DIRS, 1, RQ, RS>(st.B, st.A, st.Q, st.Sv, st.lim, nb, st.bits);
}

template <int C, bool EU, bool DIRS, int RQ, int RS>
__device__ __forceinline__ void step_even(PairLane<C>& st, const float* sq, int L, int G, int l,
                                          bool shift) {
    if (shift) {
        constexpr int slot = (C - RQ) % C;  // = (C - 1 - (RQ - 1)) mod C
        const float v = __shfl_up_sync(kFull, st.Q[slot], 1, G);
        st.Q[slot] = (l == 0) ? st.pq : v;
        if (l == 0) {
            ++st.iq;
            st.pq = st.iq + 1 < L ? __ldg(sq + st.iq + 1) : 0.f;
        }
    }
    float nb = __shfl_up_sync(kFull, st.B[C - 1], 1, G);
    if (l == 0) nb = CDTW_INF;
    dp_cells<C, EU, DIRS, 0, RQ, RS>(st.A, st.B, st.Q, st.Sv, st.lim, nb, st.bits);
}

// 2C steps (C odd/even pairs) starting with an odd step at k; rotations
// return to 0 at the end.  CHK: stop at K (else the caller guarantees
// k + 2C <= K).
template <int C, bool EU, int DM, bool CHK, int R>
__device__ __forceinline__ void body(PairLane<C>& st, const float* sq, const float* ss,
                                     uint32_t* drow, int L, int G, int l, int& k, int K,
                                     bool live) {
    if constexpr (R < C) {
        constexpr bool DIRS = DM == 1 || DM == 2;
        if (CHK && k >= K) return;
        step_odd<C, EU, DIRS, R, R + 1>(st, ss, L, G, l, true);
        store_dirs<C, DM>(st, drow, G, l, k, live);
        ++k;
        if (CHK && k >= K) return;
        step_even<C, EU, DIRS, R + 1, R + 1>(st, sq, L, G, l, true);
        store_dirs<C, DM>(st, drow, G, l, k, live);
        ++k;
        body<C, EU, DM, CHK, R + 1>(st, sq, ss, drow, L, G, l, k, K, live);
    }
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

constexpr int kWalkStages = 4;            // direction chunks in flight during backtracking
constexpr int kMoveLog = 256;             // bytes: the moves of one chunk (<= kWalkChunk)
constexpr size_t kSharedRecMax = 76 * 1024;  // shared-record mode: bytes per block (3 per SM)

// Row runs (a_i, b_i) and column runs (c_j, d_j) of the moves mlog[m0 ..
// m0 + nmax) of the group, lane l taking V consecutive moves; (gi, gj) is the
// (group-uniform) cell before move m0 and is advanced past the moves.  Every
// lane of the warp calls with the same nmax (full-mask shuffles).
template <int V>
__device__ __forceinline__ void runs_from_moves(const uint8_t* mlog, int nm, int nmax, int G,
                                                int l, bool live, int L, uint16_t* r16,
                                                uint16_t* c16, int& gi, int& gj) {
    for (int m0 = 0; m0 < nmax; m0 += V * G) {
        uint32_t bv[V];
        int nr = 0, nc = 0;
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const int m = m0 + V * l + v;
            bv[v] = m < nm ? mlog[m] : 4u;  // 4: no move
            nr += (bv[v] != 0u && bv[v] != 4u) ? 1 : 0;  // leaves its row
            nc += (bv[v] != 2u && bv[v] != 4u) ? 1 : 0;  // leaves its column
        }
        int sr = nr, sc = nc;  // inclusive scans over the group
        for (int o = 1; o < G; o <<= 1) {
            const int tr = __shfl_up_sync(kFull, sr, o, G);
            const int tc = __shfl_up_sync(kFull, sc, o, G);
            if (l >= o) {
                sr += tr;
                sc += tc;
            }
        }
        int ib = gi - (sr - nr), jb = gj - (sc - nc);  // cell before this lane's first move
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const uint32_t b = bv[v];
            const int lr = (b != 0u && b != 4u) ? 1 : 0;
            const int lc = (b != 2u && b != 4u) ? 1 : 0;
            const bool inside = live && (unsigned)ib < (unsigned)L && (unsigned)jb < (unsigned)L;
            if (inside && lr) {
                r16[2 * ib] = (uint16_t)jb;                               // a_i
                if (ib > 0) r16[2 * (ib - 1) + 1] = (uint16_t)(jb - lc);  // b_(i-1)
            }
            if (inside && lc) {
                c16[2 * jb] = (uint16_t)ib;                               // c_j
                if (jb > 0) c16[2 * (jb - 1) + 1] = (uint16_t)(ib - lr);  // d_(j-1)
            }
            ib -= lr;
            jb -= lc;
        }
        gi -= __shfl_sync(kFull, sr, G - 1, G);
        gj -= __shfl_sync(kFull, sc, G - 1, G);
    }
}

// One walker move from slot c of lane lw on anti-diagonal kw (parity e) by
// code b: diagonal keeps the slot, up (d + 1) / left (d - 1) move to slot
// c + e / c + e - 1 of the other parity.  Branch-free (the walkers of a warp
// take different moves).
template <int C>
__device__ __forceinline__ void walk_move(uint32_t b, int& kw, int& e, int& lw, int& c) {
    const bool dg = b & 1u;
    int cn = c + (dg ? 0 : (b ? e : e - 1));
    kw -= dg ? 2 : 1;
    e ^= dg ? 0 : 1;
    const bool hi = cn >= C, lo = cn < 0;
    cn += hi ? -C : (lo ? C : 0);
    lw += hi ? 1 : (lo ? -1 : 0);
    c = cn;
}

// Backtracking with the record in shared memory (DM 2): lane 0 of the group
// walks the whole record into the move log, reading the three possible next
// elements while it decodes the current one; then the group builds the runs.
template <int C>
__device__ __forceinline__ void walk_shared(const PairArgs& a, unsigned char* smem,
                                            const uint32_t* drow, int64_t pr, int L, int K,
                                            int G, int l, int gib, int e0, int porg, bool live) {
    using DT = DirT<C>;
    const DT* rec = (const DT*)drow;
    uint8_t* mlog = smem + (size_t)(blockDim.x >> a.lgG) * a.recb + (size_t)gib * a.logb;
    uint16_t* r16 = (uint16_t*)(a.rows + pr * L);  // [2i] = a_i, [2i+1] = b_i
    uint16_t* c16 = (uint16_t*)(a.cols + pr * L);  // [2j] = c_j, [2j+1] = d_j
    __syncwarp();  // the group's record is visible to its walker
    int nm = 0;
    if (l == 0 && live) {
        r16[2 * (L - 1) + 1] = (uint16_t)(L - 1);
        c16[2 * (L - 1) + 1] = (uint16_t)(L - 1);
        int kw = K - 1, e = e0, lw = porg / C, c = porg - lw * C;
        uint32_t cur = rec[(size_t)kw * G + lw];
        // every move lowers kw, so at most K moves (the log holds K bytes)
        while (kw >= 0 && (unsigned)lw < (unsigned)G) {
            const int r1 = max(kw - 1, 0), r2 = max(kw - 2, 0);
            const uint32_t n2 = rec[r2 * G + lw];
            const uint32_t n1 = rec[r1 * G + lw];
            const uint32_t n1m = rec[r1 * G + max(lw - 1, 0)];
            const uint32_t n1p = rec[r1 * G + min(lw + 1, G - 1)];
            const uint32_t b = (cur >> (2 * c)) & 3u;
            mlog[nm++] = (uint8_t)b;
            const int lw0 = lw;
            walk_move<C>(b, kw, e, lw, c);
            cur = (b & 1u) ? n2 : (lw > lw0 ? n1p : (lw < lw0 ? n1m : n1));
        }
    }
    nm = __shfl_sync(kFull, nm, 0, G);
    const int nmax = __reduce_max_sync(kFull, (unsigned)nm);
    __syncwarp();
    int gi = L - 1, gj = L - 1;
    runs_from_moves<4>(mlog, nm, nmax, G, l, live, L, r16, c16, gi, gj);
}

// Backtracking with the record in global scratch (DM 1): the record streams
// into a kWalkStages-deep shared-memory ring in chunks of R anti-diagonals
// (kWalkChunk bytes per lane, 16-byte cp.async copies), last chunk first;
// lane 0 of the group decodes a chunk's moves into a byte log (2-bit codes: 1
// or 3 diagonal, 2 up (i-1, j), 0 left (i, j-1)) and the group turns the log
// into runs.  Cell (0, 0) always records a diagonal move (its diagonal is the
// origin, the other predecessors are +inf): it writes the last runs and ends
// the walk.
template <int C>
__device__ __forceinline__ void walk_ring(const PairArgs& a, unsigned char* smem,
                                          const uint32_t* drow, int64_t pr, int L, int K, int G,
                                          int l, int gib, int e0, int porg, bool live) {
    using DT = DirT<C>;
    constexpr int R = kWalkChunk / (int)sizeof(DT);  // anti-diagonals per chunk
    unsigned char* ring = smem + (size_t)gib * kWalkStages * kWalkChunk * G;
    uint8_t* mlog = smem + (size_t)blockDim.x * kWalkStages * kWalkChunk + gib * kMoveLog;
    const int nch = (K + R - 1) / R;  // the record holds nch whole chunks per pair
    const unsigned char* rec = (const unsigned char*)drow;
    auto issue = [&](int ch) {
        if (ch < nch) {
            unsigned char* dst = ring + (ch % kWalkStages) * kWalkChunk * G;
            const unsigned char* src = rec + (size_t)(nch - 1 - ch) * kWalkChunk * G;
#pragma unroll 4
            for (int t = l; t < kWalkChunk / 16 * G; t += G) cp_async16(dst + 16 * t, src + 16 * t);
        }
        cp_async_commit();
    };
    __syncwarp();  // the group's direction elements are visible to all its lanes
#pragma unroll
    for (int ch = 0; ch < kWalkStages - 1; ++ch) issue(ch);
    uint16_t* r16 = (uint16_t*)(a.rows + pr * L);  // [2i] = a_i, [2i+1] = b_i
    uint16_t* c16 = (uint16_t*)(a.cols + pr * L);  // [2j] = c_j, [2j+1] = d_j
    if (l == 0 && live) {
        r16[2 * (L - 1) + 1] = (uint16_t)(L - 1);
        c16[2 * (L - 1) + 1] = (uint16_t)(L - 1);
    }
    int kw = K - 1, e = e0;                  // walker: anti-diagonal and its parity
    int lw = porg / C, c = porg - lw * C;    // slot c of lane lw
    int gi = L - 1, gj = L - 1;  // (group-uniform) cell before the chunk's first move
    for (int ch = 0; ch < nch; ++ch) {  // same trip count in every group of the warp
        issue(ch + kWalkStages - 1);
        cp_async_wait<kWalkStages - 1>();
        __syncwarp();
        int nm = 0;
        if (l == 0 && live) {  // groups past the last pair do not walk
            const DT* buf = (const DT*)(ring + (ch % kWalkStages) * kWalkChunk * G);
            const int rlo = (nch - 1 - ch) * R;
            // every move lowers kw: at most R (<= kMoveLog) moves per chunk
            while (kw >= rlo && (unsigned)lw < (unsigned)G) {
                const uint32_t b = ((uint32_t)buf[(kw - rlo) * G + lw] >> (2 * c)) & 3u;
                mlog[nm++] = (uint8_t)b;
                walk_move<C>(b, kw, e, lw, c);
            }
        }
        nm = __shfl_sync(kFull, nm, 0, G);
        // every lane of the warp runs the same number of scan rounds (the
        // groups' move counts differ): the full-mask shuffles below need it
        const int nmax = __reduce_max_sync(kFull, (unsigned)nm);
        __syncwarp();
        runs_from_moves<1>(mlog, nm, nmax, G, l, live, L, r16, c16, gi, gj);
        __syncwarp();
    }
    cp_async_wait<0>();
}

// Lane state at anti-diagonal 0 (D[-1][-1] = 0 under d = 0) and the first
// one or two steps, up to the first step of parity 1 (k0 = 1 or 2), where the
// bodies of 2C steps begin.  Returns k0.
template <int C, bool EU, int DM>
__device__ __forceinline__ int pair_begin(PairLane<C>& st, const float* sq, const float* ss,
                                          uint32_t* drow, int L, int W, int G, int l, int K,
                                          bool live) {
    constexpr bool DIRS = DM == 1 || DM == 2;
    const int e0 = W & 1;
    const int p0 = l * C;
    const int porg = W >> 1;  // slot of d = 0 on every anti-diagonal of parity e0
#pragma unroll
    for (int c = 0; c < C; ++c) {
        const int p = p0 + c;
        st.lim[c] = (p == W) ? CDTW_INF : -CDTW_INF;
        const float org = (p == porg) ? 0.f : CDTW_INF;  // D[-1][-1] = 0 at k = -2
        st.A[c] = e0 == 0 ? org : CDTW_INF;
        st.B[c] = e0 == 0 ? CDTW_INF : org;
        const int d = -W + 2 * p + e0;
        const int i = -d / 2, j = d / 2;  // k = 0
        st.Q[c] = (i >= 0 && i < L) ? __ldg(sq + i) : 0.f;
        st.Sv[c] = (j >= 0 && j < L) ? __ldg(ss + j) : 0.f;
    }
    st.bits = 0;
    st.iq = (W - e0) / 2;                      // lane 0's slot-0 query index at k = 0
    st.js = (-W + 2 * (G * C - 1) + e0) / 2;  // lane G-1's last-slot subject index
    st.pq = (st.iq + 1 < L) ? __ldg(sq + st.iq + 1) : 0.f;
    st.ps = (st.js + 1 < L) ? __ldg(ss + st.js + 1) : 0.f;
    int k = 0;
    if (e0 == 0) {
        step_even<C, EU, DIRS, 0, 0>(st, sq, L, G, l, false);
        store_dirs<C, DM>(st, drow, G, l, k, live);
        k = 1;
    } else {
        step_odd<C, EU, DIRS, 0, 0>(st, ss, L, G, l, false);
        store_dirs<C, DM>(st, drow, G, l, k, live);
        k = 1;
        if (k < K) {
            // query shift with the rotation kept at 0: move the window down
            const float v = __shfl_up_sync(kFull, st.Q[C - 1], 1, G);
#pragma unroll
            for (int c = C - 1; c > 0; --c) st.Q[c] = st.Q[c - 1];
            st.Q[0] = (l == 0) ? st.pq : v;
            if (l == 0) {
                ++st.iq;
                st.pq = st.iq + 1 < L ? __ldg(sq + st.iq + 1) : 0.f;
            }
            step_even<C, EU, DIRS, 0, 0>(st, sq, L, G, l, false);
            store_dirs<C, DM>(st, drow, G, l, k, live);
            k = 2;
        }
    }
    return k;
}

// Checkpoint s of a pair: the lane's two newest anti-diagonals at the start
// of a body (A = k-1, B = k-2), slot-major so a group's lanes write adjacent
// words.
template <int C>
__device__ __forceinline__ void ckpt_store(const PairLane<C>& st, float* ck, int G, int l,
                                           bool live) {
    if (!live) return;
#pragma unroll
    for (int c = 0; c < C; ++c) {
        ck[(size_t)c * G + l] = st.A[c];
        ck[(size_t)(C + c) * G + l] = st.B[c];
    }
}

// Lane state at the start of the body whose first step is k (parity 1),
// from checkpoint ck: the DP values, and the query / subject windows of step
// k-1 (rotation 0) rebuilt from the series -- the values the forward held
// there, so the recomputation is bit-identical.
template <int C>
__device__ __forceinline__ void ckpt_restore(PairLane<C>& st, const float* ck, const float* sq,
                                             const float* ss, int L, int W, int G, int l, int k) {
    const int p0 = l * C;
    const int km = k - 1;                 // last anti-diagonal computed (parity 0)
    const int em = (km + W) & 1;          // = 0
#pragma unroll
    for (int c = 0; c < C; ++c) {
        const int p = p0 + c;
        st.lim[c] = (p == W) ? CDTW_INF : -CDTW_INF;
        st.A[c] = ck[(size_t)c * G + l];
        st.B[c] = ck[(size_t)(C + c) * G + l];
        const int d = -W + 2 * p + em;
        const int i = (km - d) / 2, j = (km + d) / 2;
        st.Q[c] = (i >= 0 && i < L) ? __ldg(sq + i) : 0.f;
        st.Sv[c] = (j >= 0 && j < L) ? __ldg(ss + j) : 0.f;
    }
    st.bits = 0;
    st.iq = (km + W - em) / 2;                            // lane 0, slot 0 at k-1
    st.js = (km - W + 2 * (G * C - 1) + em) / 2;          // lane G-1, last slot at k-1
    st.pq = (st.iq + 1 < L) ? __ldg(sq + st.iq + 1) : 0.f;
    st.ps = (st.js + 1 < L) ? __ldg(ss + st.js + 1) : 0.f;
}

// DM: 0 distance only; 1 path record in global scratch, walked through a
// shared-memory ring; 2 path record in shared memory (short pairs, C <= 4);
// 3 distance plus checkpoints every a.seg anti-diagonals (the path is then
// recovered by pair_ckpt_walk_kernel).
template <int C, bool EU, int DM>
__global__ void __launch_bounds__(kPairThreads, 4) pair_fwd_kernel(const PairArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    int64_t np = a.n;  // pairs present
    if (a.gate) {
        const int c = *a.gate;
        if (c > a.gate_max || c <= a.gate_min) return;  // uniform for the whole launch
        np = min(np, (int64_t)max(c, 0));
    }
    const int G = a.G, L = a.L, W = a.W;
    const int tid = threadIdx.x;
    const int l = tid & (G - 1);
    const int gib = tid >> a.lgG;  // group in block
    const int64_t grp = (int64_t)blockIdx.x * (blockDim.x >> a.lgG) + gib;
    // a warp whose groups all lie past the pairs present has nothing to do
    // (groups never straddle warps: G is a power of two <= 32)
    if ((int64_t)blockIdx.x * (blockDim.x >> a.lgG) + ((tid & ~31) >> a.lgG) >= np) return;
    const bool live = grp < np;
    const int64_t pr = live ? grp : np - 1;
    const float* sq = a.zq + pr * a.qstride;  // the pair's series (L2-resident; edge lanes read them)
    const float* ss = a.zs + pr * L;

    const int K = 2 * L - 1;
    const int e0 = W & 1;
    const int p0 = l * C;
    const int porg = W >> 1;  // slot of d = 0 on every anti-diagonal of parity e0
    PairLane<C> st;
    uint32_t* drow = DM == 1   ? a.dirs + (size_t)pr * a.dstride
                     : DM == 2 ? (uint32_t*)(smem + (size_t)gib * a.recb)
                               : nullptr;
    int k = pair_begin<C, EU, DM>(st, sq, ss, drow, L, W, G, l, K, live);
    const int k0 = k;
    float* ck = DM == 3 ? a.ckpt + (size_t)pr * a.nseg * 2 * C * G : nullptr;
    while (k + 2 * C <= K) {
        if constexpr (DM == 3) {
            if (k > k0 && (k - k0) % a.seg == 0)
                ckpt_store<C>(st, ck + (size_t)((k - k0) / a.seg) * 2 * C * G, G, l, live);
        }
        body<C, EU, DM, false, 0>(st, sq, ss, drow, L, G, l, k, K, live);
    }
    if (k < K) {
        if constexpr (DM == 3) {
            if (k > k0 && (k - k0) % a.seg == 0)
                ckpt_store<C>(st, ck + (size_t)((k - k0) / a.seg) * 2 * C * G, G, l, live);
        }
        body<C, EU, DM, true, 0>(st, sq, ss, drow, L, G, l, k, K, live);
    }

    // D[L-1][L-1]: slot porg of the last anti-diagonal (parity e0)
    float dval = CDTW_INF;
#pragma unroll
    for (int c = 0; c < C; ++c)
        if (p0 + c == porg) dval = (e0 == 0) ? st.A[c] : st.B[c];
    if (live && p0 <= porg && porg < p0 + C) a.D[pr] = dval;
    if constexpr (DM == 1) {
        walk_ring<C>(a, smem, drow, pr, L, K, G, l, gib, e0, porg, live);
    } else if constexpr (DM == 2) {
        walk_shared<C>(a, smem, drow, pr, L, K, G, l, gib, e0, porg, live);
    }
}

// Path recovery of the checkpointed mode: per pair, the segments of a.seg
// anti-diagonals from the last to the first are recomputed from their
// checkpoints (segment 0 from the start) with direction bits into shared
// memory, and lane 0 of the group walks the path back through each segment
// as walk_ring does through its chunks; the group turns each segment's moves
// into row and column runs.  Shared memory per group: a.recb bytes of
// directions (seg x G elements) and a.logb bytes of move log (>= seg).
template <int C, bool EU>
__global__ void __launch_bounds__(kPairThreads, 4) pair_ckpt_walk_kernel(const PairArgs a) {
    using DT = DirT<C>;
    extern __shared__ __align__(16) unsigned char smem[];
    const int64_t np = a.n;
    const int G = a.G, L = a.L, W = a.W;
    const int tid = threadIdx.x;
    const int l = tid & (G - 1);
    const int gib = tid >> a.lgG;
    const int64_t grp = (int64_t)blockIdx.x * (blockDim.x >> a.lgG) + gib;
    if ((int64_t)blockIdx.x * (blockDim.x >> a.lgG) + ((tid & ~31) >> a.lgG) >= np) return;
    const bool live = grp < np;
    const int64_t pr = live ? grp : np - 1;
    const float* sq = a.zq + pr * a.qstride;
    const float* ss = a.zs + pr * L;
    const int K = 2 * L - 1;
    const int e0 = W & 1;
    const int porg = W >> 1;
    const int k0 = (e0 == 0) ? 1 : 2;
    const float* ck = a.ckpt + (size_t)pr * a.nseg * 2 * C * G;
    DT* rec = (DT*)(smem + (size_t)gib * a.recb);
    uint8_t* mlog = smem + (size_t)(blockDim.x >> a.lgG) * a.recb + (size_t)gib * a.logb;
    uint16_t* r16 = (uint16_t*)(a.rows + pr * L);  // [2i] = a_i, [2i+1] = b_i
    uint16_t* c16 = (uint16_t*)(a.cols + pr * L);  // [2j] = c_j, [2j+1] = d_j
    if (l == 0 && live) {
        r16[2 * (L - 1) + 1] = (uint16_t)(L - 1);
        c16[2 * (L - 1) + 1] = (uint16_t)(L - 1);
    }
    int kw = K - 1, e = e0;                // walker: anti-diagonal and its parity
    int lw = porg / C, c = porg - lw * C;  // slot c of lane lw
    int gi = L - 1, gj = L - 1;            // cell before the segment's first move
    for (int s = a.nseg - 1; s >= 0; --s) {
        const int kA = s == 0 ? 0 : k0 + s * a.seg;
        const int kB = min(k0 + (s + 1) * a.seg, K);
        // the record holds rows kA .. kB-1: store index k maps to row k - kA
        uint32_t* drow = (uint32_t*)((char*)rec - (ptrdiff_t)kA * G * (ptrdiff_t)sizeof(DT));
        PairLane<C> st;
        int k;
        if (s == 0) {
            k = pair_begin<C, EU, 2>(st, sq, ss, drow, L, W, G, l, K, live);
        } else {
            ckpt_restore<C>(st, ck + (size_t)s * 2 * C * G, sq, ss, L, W, G, l, kA);
            k = kA;
        }
        while (k + 2 * C <= kB) body<C, EU, 2, false, 0>(st, sq, ss, drow, L, G, l, k, kB, live);
        if (k < kB) body<C, EU, 2, true, 0>(st, sq, ss, drow, L, G, l, k, kB, live);
        __syncwarp();  // the segment's directions are visible to the walker
        int nm = 0;
        if (l == 0 && live) {
            // every move lowers kw: at most kB - kA (<= a.logb) moves here
            while (kw >= kA && (unsigned)lw < (unsigned)G) {
                const uint32_t b = ((uint32_t)rec[(size_t)(kw - kA) * G + lw] >> (2 * c)) & 3u;
                mlog[nm++] = (uint8_t)b;
                walk_move<C>(b, kw, e, lw, c);
            }
        }
        nm = __shfl_sync(kFull, nm, 0, G);
        const int nmax = __reduce_max_sync(kFull, (unsigned)nm);
        __syncwarp();
        runs_from_moves<4>(mlog, nm, nmax, G, l, live, L, r16, c16, gi, gj);
        __syncwarp();  // the record and the log are rewritten by the next segment
    }
}

using PairFwdK = void (*)(const PairArgs);

// dm 2 (shared record) is instantiated for C <= 4 only: the host selects it
// for records of at most 512 bytes per lane, which needs C <= 4.  dm 3 (the
// checkpointed forward) and dm 4 (its path recovery) for C >= 2: the host
// selects them only for pairs outside shared-record mode.
template <int C>
PairFwdK pick_fwd(bool eu, int dm) {
    if constexpr (C <= 4) {
        if (dm == 2) return eu ? pair_fwd_kernel<C, true, 2> : pair_fwd_kernel<C, false, 2>;
    }
    if constexpr (C >= 2) {
        if (dm == 3) return eu ? pair_fwd_kernel<C, true, 3> : pair_fwd_kernel<C, false, 3>;
        if (dm == 4) return eu ? pair_ckpt_walk_kernel<C, true> : pair_ckpt_walk_kernel<C, false>;
    }
    if (eu) return dm ? pair_fwd_kernel<C, true, 1> : pair_fwd_kernel<C, true, 0>;
    return dm ? pair_fwd_kernel<C, false, 1> : pair_fwd_kernel<C, false, 0>;
}

}  // namespace

// Forward kernels by lane width C, instantiated in pair_part0..3.cu (C 1-4,
// 5-8, 9-12, 13-16) for a parallel build.
PairFwdK pair_fwd_part0(int C, bool eu, int dm);
PairFwdK pair_fwd_part1(int C, bool eu, int dm);
PairFwdK pair_fwd_part2(int C, bool eu, int dm);
PairFwdK pair_fwd_part3(int C, bool eu, int dm);

}  // namespace cdtw
