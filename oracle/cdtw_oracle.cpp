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

int orc_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
