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
// the edge lanes reading the pair's z-normalised series from shared memory.
//
// With a path record the forward also stores 2 bits per band cell (diagonal
// predecessor is the minimum; up <= left) in device scratch and, once the
// pair is done, one lane backtracks from (L-1, L-1) to (0, 0) and writes the
// warping path as row runs [a_i, b_i] and column runs [c_j, d_j].  Backward
// sums the cost derivatives over those runs and applies the z-normalisation
// Jacobian (I - 11'/L - zz'/L) / sigma.
#include "common.cuh"

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

// One anti-diagonal of parity E: X (slots of k-2) becomes k from Y (k-1).
// Logical query value of slot c is Q[(c - RQ) mod C], subject value
// Sv[(c + RS) mod C].
template <int C, bool EU, bool DIRS, int E, int RQ, int RS>
__device__ __forceinline__ void dp_cells(float (&X)[C], const float (&Y)[C], const float (&Q)[C],
                                         const float (&Sv)[C], const float (&lim)[C], float nb,
                                         uint32_t& bits) {
    uint32_t nbits = 0;
#pragma unroll
    for (int c = 0; c < C; ++c) {
        const float up = (E == 0) ? Y[c] : (c == C - 1 ? nb : Y[c + 1 < C ? c + 1 : c]);
        const float left = (E == 0) ? (c == 0 ? nb : Y[c > 0 ? c - 1 : 0]) : Y[c];
        const float diag = X[c];
        const float m = min3f(diag, up, left);
        const float df = __fsub_rn(Q[(c - RQ % C + C) % C], Sv[(c + RS) % C]);
        float v = EU ? __fmaf_rn(df, df, m) : __fadd_rn(fabsf(df), m);
        if (E == 1) v = fmaxf(v, lim[c]);  // d = W + 1 lies outside the band
        X[c] = v;
        if (DIRS) {
            nbits |= (diag == m ? 1u : 0u) << (2 * c);
            nbits |= (up <= left ? 2u : 0u) << (2 * c);
        }
    }
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
            st.ps = st.js + 1 < L ? ss[st.js + 1] : 0.f;
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
            st.pq = st.iq + 1 < L ? sq[st.iq + 1] : 0.f;
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

template <int C, bool EU, bool DIRS>
__global__ void __launch_bounds__(kPairThreads) pair_fwd_kernel(const PairArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int G = a.G, L = a.L, W = a.W;
    const int tid = threadIdx.x;
    const int l = tid & (G - 1);
    const int gib = tid >> a.lgG;  // group in block
    const int64_t grp = (int64_t)blockIdx.x * (blockDim.x >> a.lgG) + gib;
    const bool live = grp < a.n;
    const int64_t pr = live ? grp : a.n - 1;
    const size_t gbytes = (size_t)round_up(8 * (int64_t)L + 64 * G, 16);
    float* sq = (float*)(smem + gib * gbytes);
    float* ss = sq + L;
    uint32_t* wbuf = (uint32_t*)(ss + L);  // kWalkRows x G words
    for (int t = l; t < L; t += G) {
        sq[t] = __ldg(a.zq + pr * L + t);
        ss[t] = __ldg(a.zs + pr * L + t);
    }
    __syncwarp();

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
        st.Q[c] = (i >= 0 && i < L) ? sq[i] : 0.f;
        st.Sv[c] = (j >= 0 && j < L) ? ss[j] : 0.f;
    }
    st.bits = 0;
    st.u = 0;
    st.kb = 0;
    st.iq = (W - e0) / 2;                      // lane 0's slot-0 query index at k = 0
    st.js = (-W + 2 * (G * C - 1) + e0) / 2;  // lane G-1's last-slot subject index
    st.pq = (st.iq + 1 < L) ? sq[st.iq + 1] : 0.f;
    st.ps = (st.js + 1 < L) ? ss[st.js + 1] : 0.f;
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
                st.pq = st.iq + 1 < L ? sq[st.iq + 1] : 0.f;
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

    // Backtracking: direction rows staged kWalkRows at a time; lane 0 walks.
    __syncwarp();
    constexpr int S = 16 / C;
    uint16_t* prow = (uint16_t*)sq;  // path runs, staged (the series are no longer needed)
    uint16_t* pcol = prow + 2 * L;
    int wi = L - 1, wj = L - 1, wk = K - 1;
    bool done = false;
    if (l == 0) {
        prow[2 * wi + 1] = (uint16_t)wj;
        pcol[2 * wj + 1] = (uint16_t)wi;
    }
    for (int rhi = a.nkb - 1; rhi >= 0; rhi -= kWalkRows) {
        __syncwarp();
#pragma unroll 4
        for (int t = 0; t < kWalkRows; ++t) {
            const int r = rhi - t;
            if (r >= 0) wbuf[t * G + l] = drow[(size_t)r * G + l];
        }
        __syncwarp();
        if (l == 0) {
            const int rlo = rhi - kWalkRows + 1;
            while (!done) {
                const int kb = wk / S;
                if (kb < rlo) break;
                if (wi == 0 && wj == 0) {
                    prow[0] = 0;
                    pcol[0] = 0;
                    done = true;
                    break;
                }
                const int e = (wk + W) & 1;
                const int p = (wj - wi + W - e) >> 1;
                const int lw = p / C, c = p - lw * C;
                const int uu = wk - kb * S;
                const uint32_t wd = wbuf[(rhi - kb) * G + lw];
                const uint32_t b = (wd >> (2 * C * (S - 1 - uu) + 2 * c)) & 3u;
                if (b & 1u) {  // diagonal
                    prow[2 * wi] = (uint16_t)wj;
                    pcol[2 * wj] = (uint16_t)wi;
                    --wi;
                    --wj;
                    wk -= 2;
                    prow[2 * wi + 1] = (uint16_t)wj;
                    pcol[2 * wj + 1] = (uint16_t)wi;
                } else if (b & 2u) {  // up: (i-1, j)
                    prow[2 * wi] = (uint16_t)wj;
                    --wi;
                    wk -= 1;
                    prow[2 * wi + 1] = (uint16_t)wj;
                } else {  // left: (i, j-1)
                    pcol[2 * wj] = (uint16_t)wi;
                    --wj;
                    wk -= 1;
                    pcol[2 * wj + 1] = (uint16_t)wi;
                }
            }
        }
    }
    __syncwarp();
    if (live) {
        const uint32_t* r32 = (const uint32_t*)prow;
        const uint32_t* c32 = (const uint32_t*)pcol;
        for (int t = l; t < L; t += G) {
            a.rows[pr * L + t] = r32[t];
            a.cols[pr * L + t] = c32[t];
        }
    }
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

// Backward: one warp per pair.  g_q[i] = sum over the row run of f'(zq_i -
// zs_j), g_s[j] = -sum over the column run; then through the z-normalisation
// and scaled by dD.
template <bool EU>
__global__ void pair_bwd_kernel(const float* __restrict__ q, const float* __restrict__ s,
                                int64_t n, int L, const double* __restrict__ hdr,
                                const uint32_t* __restrict__ rows,
                                const uint32_t* __restrict__ cols, const float* __restrict__ dD,
                                float* __restrict__ dq, float* __restrict__ ds) {
    const int lane = threadIdx.x & 31;
    const int64_t pr = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (pr >= n) return;
    const bool zn = hdr != nullptr;
    double muq = 0.0, invq = 1.0, mus = 0.0, invs = 1.0;
    bool degq = false, degs = false;
    if (zn) {
        muq = hdr[pr * 4 + 0];
        const double sq = hdr[pr * 4 + 1];
        mus = hdr[pr * 4 + 2];
        const double ssd = hdr[pr * 4 + 3];
        degq = sq < 0.0;
        degs = ssd < 0.0;
        invq = 1.0 / (degq ? 1.0 : sq);
        invs = 1.0 / (degs ? 1.0 : ssd);
    }
    const float* xq = q + pr * L;
    const float* xs = s + pr * L;
    auto zqv = [&](int t) { return zn ? pair_z(__ldg(xq + t), muq, invq) : __ldg(xq + t); };
    auto zsv = [&](int t) { return zn ? pair_z(__ldg(xs + t), mus, invs) : __ldg(xs + t); };
    auto fp = [](float df) {
        return EU ? 2.0f * df : (df > 0.f ? 1.0f : (df < 0.f ? -1.0f : 0.0f));
    };
    const float up = dD ? __ldg(dD + pr) : 1.0f;
    for (int side = 0; side < 2; ++side) {
        float* out = side == 0 ? dq : ds;
        if (!out) continue;
        const uint32_t* run = (side == 0 ? rows : cols) + pr * L;
        double sg = 0.0, sgz = 0.0;
        for (int t = lane; t < L; t += 32) {
            const uint32_t r = __ldg(run + t);
            const int lo = (int)(r & 0xffffu), hi = (int)(r >> 16);
            const float zt = side == 0 ? zqv(t) : zsv(t);
            float g = 0.f;
            for (int u = lo; u <= hi; ++u) {
                const float other = side == 0 ? zsv(u) : zqv(u);
                g += side == 0 ? fp(__fsub_rn(zt, other)) : -fp(__fsub_rn(other, zt));
            }
            out[pr * L + t] = g;
            sg += (double)g;
            sgz += (double)g * (double)zt;
        }
        if (!zn) {
            for (int t = lane; t < L; t += 32) out[pr * L + t] *= up;
            continue;
        }
        for (int o = 16; o > 0; o >>= 1) {
            sg += __shfl_xor_sync(kFull, sg, o);
            sgz += __shfl_xor_sync(kFull, sgz, o);
        }
        const bool deg = side == 0 ? degq : degs;
        const double inv = side == 0 ? invq : invs;
        const double mg = sg / (double)L, mgz = deg ? 0.0 : sgz / (double)L;
        __syncwarp();
        for (int t = lane; t < L; t += 32) {
            const double g = (double)out[pr * L + t];
            const double zt = (double)(side == 0 ? zqv(t) : zsv(t));
            out[pr * L + t] = (float)((double)up * (g - mg - zt * mgz) * inv);
        }
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
// cells per lane for short bands, 32 lanes for long ones, and G large enough
// that a warp's staged series fit in 48 KB of shared memory.
void pair_shape(int L, int W, int* G, int* C) {
    const int slots = W + 1;
    int g = 1;
    while (g < 32 && (slots + g - 1) / g > 4) g *= 2;
    while (g < 32 && (int64_t)(32 / g) * (8 * (int64_t)L + 64 * g) > 49152) g *= 2;
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
    const size_t gbytes = (size_t)round_up(8 * (int64_t)L + 64 * G, 16);
    // threads per block: up to 128, fewer when a long series leaves no room
    int threads = kPairThreads;
    while (threads > 32 && (size_t)(threads / G) * gbytes > 160 * 1024) threads /= 2;
    const size_t smem = (size_t)(threads / G) * gbytes;
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
    const int blocks = (int)div_up(n * 32, 128);
    if (euclid)
        pair_bwd_kernel<true><<<blocks, 128, 0, h->stream>>>(q, s, n, L, hdr, rows, cols, dD, dq, ds);
    else
        pair_bwd_kernel<false><<<blocks, 128, 0, h->stream>>>(q, s, n, L, hdr, rows, cols, dD, dq, ds);
    CDTW_LAUNCH(h, "pair_bwd_kernel");
    return CDTW_OK;
}

}  // namespace cdtw
