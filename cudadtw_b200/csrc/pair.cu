// Differentiable pairwise cDTW (no reference counterpart; the DP is the
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
// predecessor is the minimum; up <= left) in device scratch and, once the
// pair is done, one lane backtracks from (L-1, L-1) to (0, 0) and writes the
// warping path as row runs [a_i, b_i] and column runs [c_j, d_j].  Backward
// sums the cost derivatives over those runs and applies the z-normalisation
// Jacobian (I - 11'/L - zz'/L) / sigma.
#include "common.cuh"

#include <utility>

namespace cdtw {

namespace {

constexpr int kPairThreads = 128;
constexpr int kWalkRows = 16;  // direction rows staged per backtracking chunk
constexpr unsigned kFull = 0xffffffffu;

struct PairArgs {
    const float* zq;      // DP inputs: n x L (z-normalised copies or the raw series)
    const float* zs;
    int64_t n;
    int L, W, G, lgG;
    float* D;             // n outputs
    uint32_t* dirs;       // per pair nkb x G words (path record only)
    int nkb;
    uint32_t* rows;       // per pair L words: a_i | b_i << 16
    uint32_t* cols;       // per pair L words: c_j | d_j << 16
};

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
    if (DIRS) bits = (2 * C >= 32) ? nbits : ((bits << (2 * C)) | nbits);
}

// State of one lane of a pair's group during the forward DP.
template <int C>
struct PairLane {
    float A[C], B[C], Q[C], Sv[C], lim[C];
    uint32_t bits;
    int u, kb;     // step within the current direction word, word row
    int iq, js;    // lane 0's slot-0 query index, lane G-1's last-slot subject index
    float pq, ps;  // the values at iq + 1 / js + 1 (the next shift's)
};

template <int C, bool DIRS>
__device__ __forceinline__ void flush_bits(PairLane<C>& st, uint32_t* drow, int G, int l, int k,
                                           int K, bool live) {
    constexpr int S = 16 / C;
    if (!DIRS) return;
    if (++st.u == S || k == K - 1) {
        uint32_t w = st.bits;
        const int pad = S - st.u;
        if (pad > 0) w <<= 2 * C * pad;
        if (live) drow[(size_t)st.kb * G + l] = w;
        st.bits = 0;
        st.u = 0;
        ++st.kb;
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
// return to 0 at the end.  Stops at K.
template <int C, bool EU, bool DIRS, int R>
__device__ __forceinline__ void body(PairLane<C>& st, const float* sq, const float* ss,
                                     uint32_t* drow, int L, int G, int l, int& k, int K,
                                     bool live) {
    if constexpr (R < C) {
        if (k >= K) return;
        step_odd<C, EU, DIRS, R, R + 1>(st, ss, L, G, l, true);
        flush_bits<C, DIRS>(st, drow, G, l, k, K, live);
        if (++k >= K) return;
        step_even<C, EU, DIRS, R + 1, R + 1>(st, sq, L, G, l, true);
        flush_bits<C, DIRS>(st, drow, G, l, k, K, live);
        ++k;
        body<C, EU, DIRS, R + 1>(st, sq, ss, drow, L, G, l, k, K, live);
    }
}

__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

constexpr int kWalkStages = 4;            // direction chunks in flight during backtracking
constexpr int kMoveLog = kWalkRows * 16;  // bytes: the moves of one chunk (<= kWalkRows * S)

template <int C, bool EU, bool DIRS>
__global__ void __launch_bounds__(kPairThreads, 4) pair_fwd_kernel(const PairArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int G = a.G, L = a.L, W = a.W;
    const int tid = threadIdx.x;
    const int l = tid & (G - 1);
    const int gib = tid >> a.lgG;  // group in block
    const int64_t grp = (int64_t)blockIdx.x * (blockDim.x >> a.lgG) + gib;
    const bool live = grp < a.n;
    const int64_t pr = live ? grp : a.n - 1;
    const float* sq = a.zq + pr * L;  // the pair's series (L2-resident; edge lanes read them)
    const float* ss = a.zs + pr * L;

    const int K = 2 * L - 1;
    const int e0 = W & 1;
    const int p0 = l * C;
    const int porg = W >> 1;  // slot of d = 0 on every anti-diagonal of parity e0
    PairLane<C> st;
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
    st.u = 0;
    st.kb = 0;
    st.iq = (W - e0) / 2;                      // lane 0's slot-0 query index at k = 0
    st.js = (-W + 2 * (G * C - 1) + e0) / 2;  // lane G-1's last-slot subject index
    st.pq = (st.iq + 1 < L) ? __ldg(sq + st.iq + 1) : 0.f;
    st.ps = (st.js + 1 < L) ? __ldg(ss + st.js + 1) : 0.f;
    uint32_t* drow = DIRS ? a.dirs + (size_t)pr * a.nkb * G : nullptr;

    int k = 0;
    if (e0 == 0) {
        step_even<C, EU, DIRS, 0, 0>(st, sq, L, G, l, false);
        flush_bits<C, DIRS>(st, drow, G, l, k, K, live);
        k = 1;
    } else {
        step_odd<C, EU, DIRS, 0, 0>(st, ss, L, G, l, false);
        flush_bits<C, DIRS>(st, drow, G, l, k, K, live);
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
            flush_bits<C, DIRS>(st, drow, G, l, k, K, live);
            k = 2;
        }
    }
    while (k < K) body<C, EU, DIRS, 0>(st, sq, ss, drow, L, G, l, k, K, live);

    // D[L-1][L-1]: slot porg of the last anti-diagonal (parity e0)
    float dval = CDTW_INF;
#pragma unroll
    for (int c = 0; c < C; ++c)
        if (p0 + c == porg) dval = (e0 == 0) ? st.A[c] : st.B[c];
    if (live && p0 <= porg && porg < p0 + C) a.D[pr] = dval;
    if (!DIRS) return;

    // Backtracking: chunks of kWalkRows direction rows stream into a
    // kWalkStages-deep shared-memory ring (cp.async).  Lane 0 of the group
    // decodes the moves of a chunk into a byte log (2-bit codes: 1 or 3
    // diagonal, 2 up (i-1, j), 0 left (i, j-1)); the group then turns the log
    // into row runs (a_i, b_i) and column runs (c_j, d_j) with a scan.  Cell
    // (0, 0) always records a diagonal move (its diagonal is the origin, the
    // other predecessors are +inf): it writes the last runs and ends the walk.
    constexpr int S = 16 / C;
    uint32_t* ring = (uint32_t*)smem + (size_t)gib * kWalkStages * kWalkRows * G;
    uint8_t* mlog = smem + (size_t)blockDim.x * kWalkStages * kWalkRows * 4 + gib * kMoveLog;
    const int nch = (a.nkb + kWalkRows - 1) / kWalkRows;
    auto issue = [&](int ch) {
        if (ch < nch) {
            uint32_t* dst = ring + (ch % kWalkStages) * kWalkRows * G;
            const int rhi = a.nkb - 1 - ch * kWalkRows;
#pragma unroll 4
            for (int t = 0; t < kWalkRows; ++t) {
                const int r = rhi - t;
                if (r >= 0) cp_async4(dst + t * G + l, drow + (size_t)r * G + l);
            }
        }
        cp_async_commit();
    };
    __syncwarp();  // the group's direction words are visible to all its lanes
#pragma unroll
    for (int ch = 0; ch < kWalkStages - 1; ++ch) issue(ch);
    uint16_t* r16 = (uint16_t*)(a.rows + pr * L);  // [2i] = a_i, [2i+1] = b_i
    uint16_t* c16 = (uint16_t*)(a.cols + pr * L);  // [2j] = c_j, [2j+1] = d_j
    if (l == 0 && live) {
        r16[2 * (L - 1) + 1] = (uint16_t)(L - 1);
        c16[2 * (L - 1) + 1] = (uint16_t)(L - 1);
    }
    int kb = (K - 1) / S, uu = (K - 1) - kb * S, e = e0;  // walker: anti-diagonal kb*S+uu
    int lw = porg / C, c = porg - lw * C;                  // slot c of lane lw, parity e
    int gi = L - 1, gj = L - 1;  // (group-uniform) cell before the chunk's first move
    for (int ch = 0; ch < nch; ++ch) {  // same trip count in every group of the warp
        issue(ch + kWalkStages - 1);
        cp_async_wait<kWalkStages - 1>();
        __syncwarp();
        int nm = 0;
        if (l == 0 && live) {  // groups past the last pair do not walk
            const uint32_t* buf = ring + (ch % kWalkStages) * kWalkRows * G;
            const int rhi = a.nkb - 1 - ch * kWalkRows;
            const int rlo = max(rhi - kWalkRows + 1, 0);
            while (kb >= rlo && (unsigned)lw < (unsigned)G && nm < kMoveLog) {
                const uint32_t wd = buf[(rhi - kb) * G + lw];
                const uint32_t b = (wd >> (2 * C * (S - 1 - uu) + 2 * c)) & 3u;
                mlog[nm++] = (uint8_t)b;
                const bool dg = b & 1u;
                const int dp = dg ? 0 : (b ? e : e - 1);  // up: d + 1, left: d - 1
                e ^= dg ? 0 : 1;
                if (S == 1) {
                    kb -= 1 + dg;
                } else {
                    uu -= 1 + dg;
                    if (uu < 0) {
                        uu += S;
                        --kb;
                    }
                }
                c += dp;
                if (c >= C) {
                    c -= C;
                    ++lw;
                } else if (c < 0) {
                    c += C;
                    --lw;
                }
            }
        }
        nm = __shfl_sync(kFull, nm, 0, G);
        // every lane of the warp runs the same number of scan rounds (the
        // groups' move counts differ): the full-mask shuffles below need it
        const int nmax = __reduce_max_sync(kFull, (unsigned)nm);
        __syncwarp();
        for (int m0 = 0; m0 < nmax; m0 += G) {
            const int m = m0 + l;
            const uint32_t b = m < nm ? mlog[m] : 2u;
            const int lr = (m < nm && b != 0u) ? 1 : 0;  // leaves its row
            const int lc = (m < nm && b != 2u) ? 1 : 0;  // leaves its column
            int sr = lr, sc = lc;                        // inclusive scans over the group
            for (int o = 1; o < G; o <<= 1) {
                const int tr = __shfl_up_sync(kFull, sr, o, G);
                const int tc = __shfl_up_sync(kFull, sc, o, G);
                if (l >= o) {
                    sr += tr;
                    sc += tc;
                }
            }
            const int ib = gi - (sr - lr), jb = gj - (sc - lc);  // cell before move m
            const bool inside = live && (unsigned)ib < (unsigned)L && (unsigned)jb < (unsigned)L;
            if (inside && lr) {
                r16[2 * ib] = (uint16_t)jb;                               // a_i
                if (ib > 0) r16[2 * (ib - 1) + 1] = (uint16_t)(jb - lc);  // b_(i-1)
            }
            if (inside && lc) {
                c16[2 * jb] = (uint16_t)ib;                               // c_j
                if (jb > 0) c16[2 * (jb - 1) + 1] = (uint16_t)(ib - lr);  // d_(j-1)
            }
            gi -= __shfl_sync(kFull, sr, G - 1, G);
            gj -= __shfl_sync(kFull, sc, G - 1, G);
        }
        __syncwarp();
    }
    cp_async_wait<0>();
}

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

using PairFwdK = void (*)(const PairArgs);

template <int C>
PairFwdK pick_fwd(bool eu, bool dirs) {
    if (eu) return dirs ? pair_fwd_kernel<C, true, true> : pair_fwd_kernel<C, true, false>;
    return dirs ? pair_fwd_kernel<C, false, true> : pair_fwd_kernel<C, false, false>;
}

PairFwdK fwd_kernel(int C, bool eu, bool dirs) {
    switch (C) {
        case 1: return pick_fwd<1>(eu, dirs);
        case 2: return pick_fwd<2>(eu, dirs);
        case 3: return pick_fwd<3>(eu, dirs);
        case 4: return pick_fwd<4>(eu, dirs);
        case 5: return pick_fwd<5>(eu, dirs);
        case 6: return pick_fwd<6>(eu, dirs);
        case 7: return pick_fwd<7>(eu, dirs);
        case 8: return pick_fwd<8>(eu, dirs);
        case 9: return pick_fwd<9>(eu, dirs);
        case 10: return pick_fwd<10>(eu, dirs);
        case 11: return pick_fwd<11>(eu, dirs);
        case 12: return pick_fwd<12>(eu, dirs);
        case 13: return pick_fwd<13>(eu, dirs);
        case 14: return pick_fwd<14>(eu, dirs);
        case 15: return pick_fwd<15>(eu, dirs);
        default: return pick_fwd<16>(eu, dirs);
    }
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

size_t pair_dirs_words(int L, int W) {
    int G, C;
    pair_shape(L, W, &G, &C);
    const int S = 16 / C;
    const int64_t nkb = div_up(2 * (int64_t)L - 1, S);
    return (size_t)nkb * G;
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
                    bool euclid, float* D, uint32_t* dirs, uint32_t* rows, uint32_t* cols) {
    int G, C;
    pair_shape(L, W, &G, &C);
    if (C > 16) return set_error(h, CDTW_EUNSUPPORTED, "pair band W=%d exceeds 511", W);
    PairArgs a;
    a.zq = zq;
    a.zs = zs;
    a.n = n;
    a.L = L;
    a.W = W;
    a.G = G;
    a.lgG = 0;
    while ((1 << a.lgG) < G) ++a.lgG;
    a.D = D;
    a.dirs = dirs;
    a.nkb = (int)div_up(2 * (int64_t)L - 1, 16 / C);
    a.rows = rows;
    a.cols = cols;
    const int threads = kPairThreads;
    // backtracking ring (kWalkStages x kWalkRows words per lane) + move log per group
    const size_t smem =
        dirs ? (size_t)threads * kWalkStages * kWalkRows * 4 + (size_t)(threads / G) * kMoveLog : 0;
    const int64_t groups_per_block = threads / G;
    const int64_t blocks = div_up(n, groups_per_block);
    if (blocks > INT32_MAX) return set_error(h, CDTW_EINVAL, "too many pairs");
    const PairFwdK k = fwd_kernel(C, euclid, dirs != nullptr);
    CDTW_CUDA(h, cudaFuncSetAttribute((const void*)k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
    k<<<(int)blocks, threads, smem, h->stream>>>(a);
    CDTW_LAUNCH(h, "pair_fwd_kernel");
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
