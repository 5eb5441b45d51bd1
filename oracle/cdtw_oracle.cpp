// CPU ORACLE -- TEST INFRASTRUCTURE ONLY.
//
// This file restates, in plain FP64 C++, the arithmetic of the CUDA-DTW
// reference (gravitino/cudadtw) for the z-normalised subsequence search under
// a Sakoe-Chiba band.  It is the checker for the CUDA product path: only the
// tests, __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm
// load it.  Nothing in the cudadtw_b200 package links or calls it.
//
// Parity pins: the search result (location, distance) of this oracle is
// checked against UCR_DTW_BIN / UCR_ED_BIN built from the reference's own
// sources (oracle/Makefile -> oracle/_ref/) on the golden fixtures in
// tests/golden/.  The LB_Kim / LB_Keogh / LDTW restatements have no golden
// vectors in the reference; they are checked by the reference's own property
// tests (LB <= cDTW, tests/test_dtwbounds.cu:129-149) and by the tie rules
// stated below.
//
// Every function cites the reference file:line it follows (paths relative to
// the reference project root).

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <limits>
#include <omp.h>

namespace {

const double kInf = std::numeric_limits<double>::infinity();

inline double sq(double v) { return v * v; }

// Window statistics of one window, two-pass FP64.  The reference takes
// mu_i = (P[i+M]-P[i])/M and sigma_i = sqrt(E[x^2]-mu^2), sigma=1 when the
// variance is not positive (include/stats.cuh:30-52); UCR takes the same
// population sigma (UCR Suite/UCR_DTW_BIN.cpp:633-635).  Two passes give the
// exact-math value both approximate.
inline void window_stats(const float* x, int M, double* mu, double* sigma) {
    double s = 0.0;
    for (int k = 0; k < M; ++k) s += (double)x[k];
    const double m = s / M;
    double v = 0.0;
    for (int k = 0; k < M; ++k) v += sq((double)x[k] - m);
    v /= M;
    *mu = m;
    *sigma = v > 0.0 ? std::sqrt(v) : 1.0;
}

// Banded DTW between two equal-length sequences a (data, rows) and b (query,
// columns), |i-j| <= W, squared-Euclidean or absolute cell cost.  Same
// recurrence and band as sequential_cdtw (include/cdtw.cuh:24-88) and UCR
// dtw() without early abandoning (UCR Suite/UCR_DTW_BIN.cpp:288-354).
double banded_dtw(const double* a, const double* b, int M, int W, bool euclid,
                  std::vector<double>& prev, std::vector<double>& cur) {
    // prev/cur indexed by column j in [0, M); value of row i-1 / i.
    prev.assign(M, kInf);
    cur.assign(M, kInf);
    for (int i = 0; i < M; ++i) {
        const int lo = std::max(0, i - W), hi = std::min(M - 1, i + W);
        if (lo > 0) cur[lo - 1] = kInf;
        for (int j = lo; j <= hi; ++j) {
            const double d = a[i] - b[j];
            const double c = euclid ? d * d : std::fabs(d);
            double m;
            if (i == 0 && j == 0) m = 0.0;
            else {
                const double left = (j > lo) ? cur[j - 1] : kInf;
                const double up = (i > 0 && j <= std::min(M - 1, i - 1 + W)) ? prev[j] : kInf;
                const double diag = (i > 0 && j > 0 && j - 1 >= std::max(0, i - 1 - W)) ? prev[j - 1] : kInf;
                m = std::min(left, std::min(up, diag));
            }
            cur[j] = c + m;
        }
        if (hi + 1 < M) cur[hi + 1] = kInf;
        std::swap(prev, cur);
    }
    return prev[M - 1];
}

}  // namespace

extern "C" {

// z-normalise a query, FP64, population sigma (include/stats.cuh:8-28;
// UCR Suite/UCR_DTW_BIN.cpp:527-542).  Two-pass; sigma=1 if the variance is 0.
void orc_znorm(const double* q, int M, double* out) {
    double s = 0.0;
    for (int i = 0; i < M; ++i) s += q[i];
    const double mu = s / M;
    double v = 0.0;
    for (int i = 0; i < M; ++i) v += sq(q[i] - mu);
    v /= M;
    const double sd = v > 0.0 ? std::sqrt(v) : 1.0;
    for (int i = 0; i < M; ++i) out[i] = (q[i] - mu) / sd;
}

// Windowed mean / std of every length-M window of the stream
// (include/stats.cuh:115-142 avg_std; sigma rule of stats.cuh:49-50).
void orc_window_stats(const float* x, int64_t N, int M, double* mu, double* sigma) {
    const int64_t Nw = N - M + 1;
#pragma omp parallel for schedule(static)
    for (int64_t w = 0; w < Nw; ++w) window_stats(x + w, M, mu + w, sigma + w);
}

// cDTW of the z-normalised query against every window (no pruning): the
// all-windows path of tests/test_dtw.cu:98-158 with the CPU cDTW of
// include/cdtw.cuh:91-157, in FP64.  zq is the z-normalised query; the window
// is z-normalised with its own exact FP64 mean/std.  out[w] is the squared
// (Euclidean) or absolute (Manhattan) cDTW value, as the reference's Cdtw array.
void orc_cdtw_all(const double* zq, int M, const float* x, int64_t N, int W,
                  int euclid, double* out) {
    const int64_t Nw = N - M + 1;
#pragma omp parallel
    {
        std::vector<double> z(M), prev, cur;
#pragma omp for schedule(dynamic, 256)
        for (int64_t w = 0; w < Nw; ++w) {
            double mu, sd;
            window_stats(x + w, M, &mu, &sd);
            for (int k = 0; k < M; ++k) z[k] = ((double)x[w + k] - mu) / sd;
            out[w] = banded_dtw(z.data(), zq, M, W, euclid != 0, prev, cur);
        }
    }
}

// cDTW of the z-normalised query against an explicit list of windows.
void orc_cdtw_list(const double* zq, int M, const float* x, int64_t N, int W,
                   int euclid, const int64_t* idx, int64_t L, double* out) {
    (void)N;
#pragma omp parallel
    {
        std::vector<double> z(M), prev, cur;
#pragma omp for schedule(dynamic, 16)
        for (int64_t t = 0; t < L; ++t) {
            const int64_t w = idx[t];
            double mu, sd;
            window_stats(x + w, M, &mu, &sd);
            for (int k = 0; k < M; ++k) z[k] = ((double)x[w + k] - mu) / sd;
            out[t] = banded_dtw(z.data(), zq, M, W, euclid != 0, prev, cur);
        }
    }
}

// cDTW of two already-normalised sequences (used for pair / gradient checks).
double orc_cdtw_pair(const double* a, const double* b, int M, int W, int euclid) {
    std::vector<double> prev, cur;
    return banded_dtw(a, b, M, W, euclid != 0, prev, cur);
}

// First strict minimum (UCR keeps the earliest location on ties,
// UCR Suite/UCR_DTW_BIN.cpp:682-687; ldtw.cuh:177-192 determine_min).
void orc_argmin(const double* v, int64_t n, int64_t* idx, double* val) {
    double best = kInf;
    int64_t bi = -1;
    for (int64_t i = 0; i < n; ++i)
        if (v[i] < best) { best = v[i]; bi = i; }
    *idx = bi;
    *val = best;
}

// Query envelope: U[i] = max q[i-W..i+W], L[i] = min q[i-W..i+W], clipped to
// [0, M).  Same output as Lemire's streaming filter (include/bounds.cuh:13-64,
// UCR Suite/UCR_DTW_BIN.cpp:129-176), computed by brute force.
void orc_envelope(const double* q, int M, int W, double* L, double* U) {
    for (int i = 0; i < M; ++i) {
        double lo = kInf, hi = -kInf;
        for (int k = std::max(0, i - W); k <= std::min(M - 1, i + W); ++k) {
            lo = std::min(lo, q[k]);
            hi = std::max(hi, q[k]);
        }
        L[i] = lo;
        U[i] = hi;
    }
}

// LB_Kim of the reference GPU path: 5x5 unconstrained DTW at the front (min
// over its last row and column) plus 5x5 DTW at the back read at the
// bottom-right cell, on the z-normalised window (include/bounds.cuh:283-407).
// Requires M >= 11 (bounds.cuh:433-437).  Costs are squared or absolute.
static double lbkim_one(const double* zq, const double* s, int M, bool euclid) {
    auto c = [&](double a, double b) { double d = a - b; return euclid ? d * d : std::fabs(d); };
    double F[5][5];
    // front block: rows = query positions 0..4, cols = window positions 0..4
    for (int r = 0; r < 5; ++r)
        for (int k = 0; k < 5; ++k) {
            double best;
            if (r == 0 && k == 0) best = 0.0;
            else if (r == 0) best = F[0][k - 1];
            else if (k == 0) best = F[r - 1][0];
            else best = std::min(F[r][k - 1], std::min(F[r - 1][k - 1], F[r - 1][k]));
            F[r][k] = c(zq[r], s[k]) + best;
        }
    double mem = kInf;
    for (int k = 0; k < 5; ++k) mem = std::min(mem, F[4][k]);
    for (int r = 0; r < 5; ++r) mem = std::min(mem, F[r][4]);
    // back block: the path may enter anywhere on its first row / column
    double B[5][5];
    for (int r = 0; r < 5; ++r)
        for (int k = 0; k < 5; ++k) {
            double best;
            if (r == 0 || k == 0) best = 0.0;
            else best = std::min(B[r][k - 1], std::min(B[r - 1][k - 1], B[r - 1][k]));
            B[r][k] = c(zq[M - 5 + r], s[M - 5 + k]) + best;
        }
    return mem + B[4][4];
}

void orc_lb_kim(const double* zq, int M, const float* x, int64_t N, int euclid, double* out) {
    const int64_t Nw = N - M + 1;
#pragma omp parallel
    {
        std::vector<double> z(M);
#pragma omp for schedule(static)
        for (int64_t w = 0; w < Nw; ++w) {
            double mu, sd;
            window_stats(x + w, M, &mu, &sd);
            for (int k = 0; k < M; ++k) z[k] = ((double)x[w + k] - mu) / sd;
            out[w] = lbkim_one(zq, z.data(), M, euclid != 0);
        }
    }
}

// LB_Keogh against the query envelope, no early exit
// (include/bounds.cuh:111-144 random_lb_keogh; squared or absolute residues).
void orc_lb_keogh(const double* zq, int M, int W, const float* x, int64_t N, int euclid,
                  double* out) {
    std::vector<double> L(M), U(M);
    orc_envelope(zq, M, W, L.data(), U.data());
    const int64_t Nw = N - M + 1;
#pragma omp parallel for schedule(static)
    for (int64_t w = 0; w < Nw; ++w) {
        double mu, sd;
        window_stats(x + w, M, &mu, &sd);
        double acc = 0.0;
        for (int k = 0; k < M; ++k) {
            const double z = ((double)x[w + k] - mu) / sd;
            const double up = z - U[k], lo = z - L[k];
            if (euclid) acc += (up > 0 ? up * up : 0.0) + (lo < 0 ? lo * lo : 0.0);
            else acc += (up > 0 ? up : 0.0) - (lo < 0 ? lo : 0.0);
        }
        out[w] = acc;
    }
}

// Reverse LB_Keogh: the query against the envelope of the data
// (UCR Suite/UCR_DTW_BIN.cpp:262-282).  As in UCR (:607, :661) the data
// envelope is the stream-wide min/max over [p-W, p+W] (clipped to the stream,
// not to the window), z-normalised with the window's statistics.
void orc_lb_keogh_rev(const double* zq, int M, int W, const float* x, int64_t N, int euclid,
                      double* out) {
    std::vector<double> Lx(N), Ux(N);
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < N; ++p) {
        double lo = kInf, hi = -kInf;
        for (int64_t k = std::max<int64_t>(0, p - W); k <= std::min<int64_t>(N - 1, p + W); ++k) {
            lo = std::min(lo, (double)x[k]);
            hi = std::max(hi, (double)x[k]);
        }
        Lx[p] = lo;
        Ux[p] = hi;
    }
    const int64_t Nw = N - M + 1;
#pragma omp parallel for schedule(static)
    for (int64_t w = 0; w < Nw; ++w) {
        double mu, sd;
        window_stats(x + w, M, &mu, &sd);
        double acc = 0.0;
        for (int k = 0; k < M; ++k) {
            const double uu = (Ux[w + k] - mu) / sd, ll = (Lx[w + k] - mu) / sd;
            double d = 0.0;
            if (zq[k] > uu) d = euclid ? sq(zq[k] - uu) : zq[k] - uu;
            else if (zq[k] < ll) d = euclid ? sq(zq[k] - ll) : ll - zq[k];
            acc += d;
        }
        out[w] = acc;
    }
}

// Greedy locally-optimal warping path in the band with z-normalisation
// (include/ldtw.cuh:74-127 z_serial_ldtw), FP64.  Tie rule exactly as the
// reference (:109-123): diag if strictly below both, else down if
// !(diag<down) and down<right, else right.  Out-of-range moves cost INFTY=1e10
// (ldtw.cuh:8).  Returns the squared (Euclidean) or absolute path cost.
static double ldtw_one(const double* zq, const double* z, int M, int W, bool euclid) {
    const double INFTY = 1e10;
    auto c = [&](double a, double b) { double d = a - b; return euclid ? d * d : std::fabs(d); };
    int i = 0, j = 0;
    double d = c(zq[0], z[0]);
    while (i + 1 != M || j + 1 != M) {
        double diag = INFTY, rght = INFTY, down = INFTY;
        if (i + 1 < M && j + 1 < M) diag = c(zq[i + 1], z[j + 1]);
        if (i + 1 < M && std::abs(i - j + 1) <= W) down = c(zq[i + 1], z[j]);
        if (j + 1 < M && std::abs(j - i + 1) <= W) rght = c(zq[i], z[j + 1]);
        const bool diagSdown = diag < down, diagSrght = diag < rght, downSrght = down < rght;
        if (diagSdown && diagSrght) { d += diag; ++i; ++j; }
        else if (!diagSdown && downSrght) { d += down; ++i; }
        else { d += rght; ++j; }
    }
    return d;
}

void orc_ldtw_all(const double* zq, int M, const float* x, int64_t N, int W, int euclid,
                  double* out) {
    const int64_t Nw = N - M + 1;
#pragma omp parallel
    {
        std::vector<double> z(M);
#pragma omp for schedule(static)
        for (int64_t w = 0; w < Nw; ++w) {
            double mu, sd;
            window_stats(x + w, M, &mu, &sd);
            for (int k = 0; k < M; ++k) z[k] = ((double)x[w + k] - mu) / sd;
            out[w] = ldtw_one(zq, z.data(), M, W, euclid != 0);
        }
    }
}

// z-normalised squared Euclidean distance of the query to every window:
// sum_k (zq_k - z_k)^2 = 2M - 2 corr/sigma (include/ed.cuh:61-69, :149-150;
// UCR Suite/UCR_ED_BIN.cpp:55-75).  FP64 stream.
void orc_ed_all(const double* zq, int M, const double* x, int64_t N, double* out) {
    const int64_t Nw = N - M + 1;
#pragma omp parallel for schedule(static)
    for (int64_t w = 0; w < Nw; ++w) {
        double s = 0.0;
        for (int k = 0; k < M; ++k) s += x[w + k];
        const double mu = s / M;
        double v = 0.0;
        for (int k = 0; k < M; ++k) v += sq(x[w + k] - mu);
        v /= M;
        const double sd = v > 0.0 ? std::sqrt(v) : 1.0;
        double acc = 0.0;
        for (int k = 0; k < M; ++k) acc += sq(zq[k] - (x[w + k] - mu) / sd);
        out[w] = acc;
    }
}

// The reference's own CPU all-windows cDTW in FP32, restated for timing the
// CPU baseline: openmp_cdtw (include/cdtw.cuh:91-157) with float arithmetic,
// (subject-avg)/std computed per cell as there, `nthreads` OpenMP threads.
// zq is the FP32 z-normalised query; avg/std are FP32 per-window stats.
void orc_cdtw_ref_f32(const float* zq, int M, const float* x, const float* avg,
                      const float* sd, const int64_t* idx, int64_t L, int W,
                      int nthreads, float* out) {
    const int lane = M + 1;
#pragma omp parallel num_threads(nthreads)
    {
        std::vector<float> penalty(2 * lane);
#pragma omp for schedule(dynamic, 64)
        for (int64_t t = 0; t < L; ++t) {
            penalty[0] = 0.0f;
            for (int m = 1; m < lane; ++m) penalty[m] = INFINITY;
            int src_row = 1, trg_row = 0;
            const int64_t w = idx[t];
            const float a = avg[w], s = sd[w];
            for (int i = 1; i < lane; ++i) {
                trg_row = src_row;
                src_row = (trg_row == 0);
                const int lower = std::max(0, i - W - 1), upper = std::min(lane, i + W + 1);
                penalty[trg_row * lane + lower] = INFINITY;
                for (int j = lower + 1; j < upper; ++j) {
                    const float v = zq[i - 1] - (x[w + j - 1] - a) / s;
                    float weight = v * v;
                    weight += std::min(penalty[src_row * lane + j - 1],
                                       std::min(penalty[src_row * lane + j],
                                                penalty[trg_row * lane + j - 1]));
                    penalty[trg_row * lane + j] = weight;
                }
                if (upper < lane) penalty[trg_row * lane + upper] = INFINITY;
            }
            out[t] = penalty[trg_row * lane + M];
        }
    }
}

// ---- pairwise cDTW forward / backward (no reference counterpart) ----------
//
// The banded DP of banded_dtw above on two equal-length series, with the
// predecessor kept per cell: diagonal if it is the minimum, else (i-1, j) if
// it is <= (i, j-1), else (i, j-1).  Backtracking from (L-1, L-1) gives the
// warping path; the (sub)gradient of D = sum over the path of cost(zq_i - zs_j)
// is the sum of cost'(zq_i - zs_j) over the path cells of row i (query) or
// column j (subject, negated), then through the z-normalisation
// z = (x - mu) / sigma: dx = (g - mean(g) - z * mean(g z)) / sigma
// (sigma = 1 and no z term when the variance is not positive).
//
// f32 = 1 replays the device arithmetic: float DP with one fused
// multiply-add per cell (|d| + m for the absolute cost), float gradient sums
// in ascending order along each run.  f32 = 0 is FP64 throughout.
// margin[p] = smallest gap (second-best minus best predecessor, relative to
// the best) over the path cells: where it is tiny a float DP may pick another
// path of (almost) equal cost.
}  // extern "C"

namespace {

template <class T, class X>
void pair_one(const X* q, const X* s, int L, int W, bool euclid, bool zn, float up_grad,
              double* Dout, double* dq, double* ds, double* margin) {
    const T inf = std::numeric_limits<T>::infinity();
    std::vector<T> a(L), b(L);
    double muq = 0, sdq = 1, mus = 0, sds = 1;
    bool degq = false, degs = false;
    auto norm = [&](const X* x, std::vector<T>& z, double& mu, double& sd, bool& deg) {
        double s1 = 0.0;
        for (int t = 0; t < L; ++t) s1 += (double)x[t];
        mu = s1 / L;
        double s2 = 0.0;
        for (int t = 0; t < L; ++t) s2 += sq((double)x[t] - mu);
        const double var = s2 / L;
        deg = !(var > 0.0);
        sd = deg ? 1.0 : std::sqrt(var);
        const double inv = 1.0 / sd;
        for (int t = 0; t < L; ++t) z[t] = (T)(((double)x[t] - mu) * inv);
    };
    if (zn) {
        norm(q, a, muq, sdq, degq);
        norm(s, b, mus, sds, degs);
    } else {
        for (int t = 0; t < L; ++t) {
            a[t] = (T)q[t];
            b[t] = (T)s[t];
        }
    }
    const int w2 = 2 * W + 1;
    std::vector<T> Dt((size_t)L * w2, inf);
    std::vector<unsigned char> dir((size_t)L * w2, 0);
    auto at = [&](int i, int j) -> T {
        if (i < 0 || j < 0 || j - i > W || i - j > W) return inf;
        return Dt[(size_t)i * w2 + (j - i + W)];
    };
    for (int i = 0; i < L; ++i) {
        for (int j = std::max(0, i - W); j <= std::min(L - 1, i + W); ++j) {
            const T diag = (i == 0 && j == 0) ? (T)0 : at(i - 1, j - 1);
            const T upv = at(i - 1, j), left = at(i, j - 1);
            const T m = std::min(diag, std::min(upv, left));
            T v;
            if (sizeof(T) == 4) {
                const float df = (float)a[i] - (float)b[j];
                v = euclid ? (T)std::fmaf(df, df, (float)m) : (T)(std::fabs(df) + (float)m);
            } else {
                const double df = (double)a[i] - (double)b[j];
                v = euclid ? (T)(df * df + (double)m) : (T)(std::fabs(df) + (double)m);
            }
            Dt[(size_t)i * w2 + (j - i + W)] = v;
            dir[(size_t)i * w2 + (j - i + W)] = diag == m ? 0 : (upv <= left ? 1 : 2);
        }
    }
    *Dout = (double)at(L - 1, L - 1);
    // backtrack: row runs [ra, rb], column runs [ca, cb]
    std::vector<int> ra(L), rb(L), ca(L), cb(L);
    int i = L - 1, j = L - 1;
    rb[i] = j;
    cb[j] = i;
    double mg = kInf;
    while (!(i == 0 && j == 0)) {
        const T diag = at(i - 1, j - 1), upv = at(i - 1, j), left = at(i, j - 1);
        T v3[3] = {diag, upv, left};
        std::sort(v3, v3 + 3);
        if (v3[1] < inf) mg = std::min(mg, ((double)v3[1] - (double)v3[0]) / std::max((double)v3[0], 1e-300));
        const int d = dir[(size_t)i * w2 + (j - i + W)];
        if (d == 0) {
            ra[i] = j;
            ca[j] = i;
            --i;
            --j;
            rb[i] = j;
            cb[j] = i;
        } else if (d == 1) {
            ra[i] = j;
            --i;
            rb[i] = j;
        } else {
            ca[j] = i;
            --j;
            cb[j] = i;
        }
    }
    ra[0] = 0;
    ca[0] = 0;
    *margin = mg;
    auto fp = [&](T df) -> T {
        return euclid ? (T)2 * df : (df > 0 ? (T)1 : (df < 0 ? (T)-1 : (T)0));
    };
    for (int side = 0; side < 2; ++side) {
        double* out = side == 0 ? dq : ds;
        std::vector<T> g(L);
        for (int t = 0; t < L; ++t) {
            T acc = 0;
            const int lo = side == 0 ? ra[t] : ca[t], hi = side == 0 ? rb[t] : cb[t];
            for (int u = lo; u <= hi; ++u)
                acc += side == 0 ? fp(a[t] - b[u]) : -fp(a[u] - b[t]);
            g[t] = acc;
        }
        const std::vector<T>& z = side == 0 ? a : b;
        if (!zn) {
            for (int t = 0; t < L; ++t) out[t] = (double)(g[t] * (T)up_grad);
            continue;
        }
        double sg = 0.0, sgz = 0.0;
        for (int t = 0; t < L; ++t) {
            sg += (double)g[t];
            sgz += (double)g[t] * (double)z[t];
        }
        const bool deg = side == 0 ? degq : degs;
        const double sd = side == 0 ? sdq : sds;
        const double m1 = sg / L, m2 = deg ? 0.0 : sgz / L;
        for (int t = 0; t < L; ++t)
            out[t] = (double)up_grad * ((double)g[t] - m1 - (double)z[t] * m2) / sd;
    }
}

}  // namespace

extern "C" {

void orc_pair_fwdbwd(const float* q, const float* s, int64_t n, int L, int W, int euclid,
                     int znorm, int f32, const float* dD, double* D, double* dq, double* ds,
                     double* margin) {
    W = std::max(0, std::min(W, L - 1));
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t p = 0; p < n; ++p) {
        const float up = dD ? dD[p] : 1.0f;
        if (f32)
            pair_one<float, float>(q + p * L, s + p * L, L, W, euclid != 0, znorm != 0, up, D + p,
                            dq + p * L, ds + p * L, margin + p);
        else
            pair_one<double, float>(q + p * L, s + p * L, L, W, euclid != 0, znorm != 0, up, D + p,
                             dq + p * L, ds + p * L, margin + p);
    }
}

// FP64 cost and gradient along a GIVEN warping path (row runs rows[i] =
// a_i | b_i << 16, column runs cols[j] = c_j | d_j << 16, the device path
// record): checks that a device path is optimal and that its gradient is the
// derivative of the cost along it.  Returns per pair 1 if the runs form a
// monotone connected path from (0, 0) to (L-1, L-1) inside the band, else 0.
void orc_pair_path_grad(const float* q, const float* s, int64_t n, int L, int W, int euclid,
                        int znorm, const uint32_t* rows, const uint32_t* cols, const float* dD,
                        double* cost, double* dq, double* ds, int* valid) {
    W = std::max(0, std::min(W, L - 1));
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t p = 0; p < n; ++p) {
        const float* x = q + p * L;
        const float* y = s + p * L;
        const uint32_t* R = rows + p * L;
        const uint32_t* Cc = cols + p * L;
        std::vector<double> a(L), b(L);
        double sd[2] = {1, 1};
        bool deg[2] = {false, false};
        for (int side = 0; side < 2; ++side) {
            const float* v = side ? y : x;
            std::vector<double>& z = side ? b : a;
            if (!znorm) {
                for (int t = 0; t < L; ++t) z[t] = v[t];
                continue;
            }
            double s1 = 0;
            for (int t = 0; t < L; ++t) s1 += v[t];
            const double mu = s1 / L;
            double s2 = 0;
            for (int t = 0; t < L; ++t) s2 += sq(v[t] - mu);
            deg[side] = !(s2 / L > 0.0);
            sd[side] = deg[side] ? 1.0 : std::sqrt(s2 / L);
            for (int t = 0; t < L; ++t) z[t] = (v[t] - mu) / sd[side];
        }
        bool ok = true;
        double c = 0;
        for (int i = 0; i < L && ok; ++i) {
            const int lo = (int)(R[i] & 0xffff), hi = (int)(R[i] >> 16);
            ok = lo <= hi && hi < L && std::abs(i - lo) <= W && std::abs(i - hi) <= W;
            if (i == 0) ok = ok && lo == 0;
            if (i == L - 1) ok = ok && hi == L - 1;
            if (i > 0) {
                const int phi = (int)(R[i - 1] >> 16);
                ok = ok && (lo == phi || lo == phi + 1);
            }
            for (int j = lo; ok && j <= hi; ++j) {
                const double d = a[i] - b[j];
                c += euclid ? d * d : std::fabs(d);
                // the column runs must describe the same cells
                const int clo = (int)(Cc[j] & 0xffff), chi = (int)(Cc[j] >> 16);
                ok = clo <= i && i <= chi;
            }
        }
        valid[p] = ok ? 1 : 0;
        cost[p] = c;
        const double up = dD ? dD[p] : 1.0;
        auto fp = [&](double d) { return euclid ? 2 * d : (d > 0 ? 1.0 : (d < 0 ? -1.0 : 0.0)); };
        for (int side = 0; side < 2; ++side) {
            double* out = (side ? ds : dq) + p * L;
            const uint32_t* run = side ? Cc : R;
            const std::vector<double>& z = side ? b : a;
            std::vector<double> g(L, 0.0);
            for (int t = 0; t < L && ok; ++t) {
                const int lo = (int)(run[t] & 0xffff), hi = (int)(run[t] >> 16);
                for (int u = lo; u <= std::min(hi, L - 1); ++u)
                    g[t] += side ? -fp(a[u] - b[t]) : fp(a[t] - b[u]);
            }
            double sg = 0, sgz = 0;
            for (int t = 0; t < L; ++t) {
                sg += g[t];
                sgz += g[t] * z[t];
            }
            const double m1 = znorm ? sg / L : 0.0;
            const double m2 = (znorm && !deg[side]) ? sgz / L : 0.0;
            for (int t = 0; t < L; ++t) out[t] = up * (g[t] - m1 - z[t] * m2) / sd[side];
        }
    }
}

// FP64 forward/backward on double inputs: the finite-difference pin of the
// backtracking gradient (central differences need steps far below float
// resolution).
void orc_pair_fwdbwd64(const double* q, const double* s, int64_t n, int L, int W, int euclid,
                       int znorm, double* D, double* dq, double* ds, double* margin) {
    W = std::max(0, std::min(W, L - 1));
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t p = 0; p < n; ++p)
        pair_one<double, double>(q + p * L, s + p * L, L, W, euclid != 0, znorm != 0, 1.0f, D + p,
                                 dq + p * L, ds + p * L, margin + p);
}

int orc_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
