// Peak cell-update rate of this GPU for the roofline of the cDTW kernels.
//
// A DTW cell update in its minimal form is three instructions: FADD (z - q),
// three-input FMNMX (min of the three predecessors) and FFMA (d*d + min).
// This kernel issues exactly that sequence on many independent chains per
// thread (no memory traffic in the loop), so its cells/s is the issue-bound
// ceiling that a cDTW kernel can approach on this part at the clocks it runs.
#include "common.cuh"

namespace cdtw {

namespace {

constexpr int kChains = 8;

__global__ void __launch_bounds__(256)
peak_cell_kernel(const float* __restrict__ seed, int iters, float* __restrict__ sink) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    float z = seed[t & 255], q = seed[(t + 7) & 255];
    float a[kChains], b[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) {
        a[c] = seed[(t + c) & 255];
        b[c] = seed[(t + 3 * c + 1) & 255];
    }
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) {
            // two independent cells per chain per iteration, each FADD + FMNMX3
            // + FFMA (independent within the iteration: the highest issue rate
            // of the update, the strictest denominator)
            const float d0 = z - a[c];
            const float m0 = min3f(a[c], b[c], q);
            const float v0 = fmaf(d0, d0, m0);
            const float d1 = q - b[c];
            const float m1 = min3f(b[c], a[c], z);
            const float v1 = fmaf(d1, d1, m1);
            a[c] = v0;  // values may grow to +inf; inf arithmetic issues at the same rate
            b[c] = v1;
        }
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += a[c] + b[c];
    if (s == 12345.678f) sink[t & 255] = s;  // keeps the work alive; sink holds 256 floats
}

}  // namespace

}  // namespace cdtw

using namespace cdtw;

extern "C" int cdtw_calibrate_cell_rate(cdtw_handle h, double* cells_per_second) {
    if (!h || !cells_per_second) return CDTW_EINVAL;
    CDTW_CUDA(h, cudaSetDevice(h->device));
    float* buf = nullptr;
    CDTW_CUDA(h, cudaMallocAsync((void**)&buf, 256 * sizeof(float) * 2, h->stream));
    float* sink = buf + 256;
    // any finite positive values
    float hv[256];
    for (int i = 0; i < 256; ++i) hv[i] = 0.25f + 0.001f * (float)i;
    CDTW_CUDA(h, cudaMemcpyAsync(buf, hv, sizeof(hv), cudaMemcpyHostToDevice, h->stream));
    const int blocks = h->sm_count * 8, threads = 256, iters = 4096;
    cudaEvent_t e0, e1;
    CDTW_CUDA(h, cudaEventCreate(&e0));
    CDTW_CUDA(h, cudaEventCreate(&e1));
    peak_cell_kernel<<<blocks, threads, 0, h->stream>>>(buf, iters, sink);  // warm-up
    CDTW_LAUNCH(h, "peak_cell_kernel");
    float best_ms = 1e30f;
    for (int r = 0; r < 5; ++r) {
        CDTW_CUDA(h, cudaEventRecord(e0, h->stream));
        peak_cell_kernel<<<blocks, threads, 0, h->stream>>>(buf, iters, sink);
        CDTW_CUDA(h, cudaEventRecord(e1, h->stream));
        CDTW_CUDA(h, cudaEventSynchronize(e1));
        float ms = 0.f;
        CDTW_CUDA(h, cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best_ms) best_ms = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    CDTW_CUDA(h, cudaFreeAsync(buf, h->stream));
    // 2 cells per chain-iteration
    const double cells = (double)blocks * threads * iters * kChains * 2.0;
    *cells_per_second = cells / (best_ms * 1e-3);
    return CDTW_OK;
}
