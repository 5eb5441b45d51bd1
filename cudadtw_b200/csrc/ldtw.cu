// Greedy locally-optimal warping path inside the Sakoe-Chiba band (LDTW),
// z-normalised, for every window: the GPU-LDTW path.
//
// Reference: ztsh2_ldtw (include/ldtw.cuh:294-391) and its serial twin
// z_serial_ldtw (ldtw.cuh:74-127): one path of at most 2M-2 steps per window;
// at (i, j) take the diagonal if it is strictly cheaper than both the cell
// below and the cell to the right, else "down" if the diagonal is not cheaper
// than it and it is cheaper than "right", else "right"; moves outside the
// matrix or the band cost INFTY = 1e10 (ldtw.cuh:8).  One thread per window
// here too (a path is inherently sequential), in FP64 so the branch decisions
// match the FP64 oracle; the four values a step reads (two query, two window
// samples) are carried in registers and only the entering ones are loaded.
#include "common.cuh"

namespace cdtw {

namespace {

template <bool EU>
__device__ __forceinline__ double lcost(double d) { return EU ? d * d : fabs(d); }

template <bool EU>
__global__ void __launch_bounds__(128)
ldtw_kernel(const float* __restrict__ x, const double* __restrict__ mu,
            const double* __restrict__ sigma, const double* __restrict__ zq, int M, int W,
            int64_t Nw, double* __restrict__ out) {
    const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= Nw) return;
    const double INFTY = 1e10;
    const double m = mu[w], s = sigma[w];
    const float* __restrict__ xw = x + w;
    int i = 0, j = 0;
    double q0 = zq[0], q1 = (M > 1) ? zq[1] : 0.0;
    double s0 = ((double)xw[0] - m) / s, s1 = (M > 1) ? ((double)xw[1] - m) / s : 0.0;
    double d = lcost<EU>(q0 - s0);
    // every step advances i or j, so 2M-2 steps reach (M-1, M-1); the cap only
    // guards against non-finite input
    for (int it = 0; it < 2 * M && (i + 1 != M || j + 1 != M); ++it) {
        double diag = INFTY, rght = INFTY, down = INFTY;
        if (i + 1 < M && j + 1 < M) diag = lcost<EU>(q1 - s1);
        if (i + 1 < M && abs(i - j + 1) <= W) down = lcost<EU>(q1 - s0);
        if (j + 1 < M && abs(j - i + 1) <= W) rght = lcost<EU>(q0 - s1);
        const bool diagSdown = diag < down, diagSrght = diag < rght, downSrght = down < rght;
        bool mi, mj;
        if (diagSdown && diagSrght) {
            d += diag;
            mi = mj = true;
        } else if (!diagSdown && downSrght) {
            d += down;
            mi = true;
            mj = false;
        } else {
            d += rght;
            mi = false;
            mj = true;
        }
        if (mi) {
            ++i;
            q0 = q1;
            q1 = (i + 1 < M) ? zq[i + 1] : 0.0;
        }
        if (mj) {
            ++j;
            s0 = s1;
            s1 = (j + 1 < M) ? ((double)xw[j + 1] - m) / s : 0.0;
        }
    }
    out[w] = d;
}

}  // namespace

int launch_ldtw(cdtw_handle h, const float* x, int64_t N, const double* mu, const double* sigma,
                bool euclid, double* out) {
    const QueryPack& q = h->q;
    const int64_t Nw = N - q.M + 1;
    const unsigned blocks = (unsigned)div_up(Nw, 128);
    if (euclid)
        ldtw_kernel<true><<<blocks, 128, 0, h->stream>>>(x, mu, sigma, q.zq64, q.M, q.W, Nw, out);
    else
        ldtw_kernel<false><<<blocks, 128, 0, h->stream>>>(x, mu, sigma, q.zq64, q.M, q.W, Nw, out);
    CDTW_LAUNCH(h, "ldtw_kernel");
    return CDTW_OK;
}

}  // namespace cdtw
