// All-windows cDTW for callers that cannot allocate device memory.
//
// The handle API allocates: cdtw_create takes pinned host memory and a
// stream, and the first call at a new size grows the handle's device work
// area with cudaMalloc.  Some callers cannot allow that: a host that owns the
// whole device memory budget and lends the library only the buffers of one
// call (a caching allocator or a plugin interface that forbids allocation in
// its callbacks), or a latency-critical pipeline where the device-wide
// synchronisation of cudaMalloc/cudaFree would stall its other streams.  For
// them cdtw_all_windows_noalloc runs the same three kernels as
// cdtw_set_query + cdtw_avg_std + cdtw_gpu_cdtw(all windows), with the query
// pack and the window statistics kept in one fixed device array defined in
// this file instead of a handle's work area.
//
// The array is a file-scope __device__ variable, so every GPU that loads the
// library holds it (CDTW_NOALLOC_SCRATCH_BYTES, about 12.3 MiB) until the
// process exits.  Host code cannot use the array's name as a device address;
// the first call on each device looks the address up with
// cudaGetSymbolAddress while that device is current and keeps it, together
// with the unique ID of the CUDA context it belongs to.  A later call in a
// different context (after cudaDeviceReset, or a released and re-created
// primary context, where the module loads again and the array may move)
// looks the address up again.
#include "common.cuh"

#include <cuda.h>  // CUcontext / CUresult types only; the driver calls are resolved at run time

#include <mutex>

namespace {

constexpr int kNoAllocMaxBand = 40;  // bands served by this entry point

constexpr size_t align256(size_t b) { return (b + 255) / 256 * 256; }

// Layout of the fixed array, sized for the largest accepted request.
constexpr size_t kLqMax = (size_t)(CDTW_NOALLOC_MAX_QUERY + 2 * (CDTW_NOALLOC_MAX_QUERY - 1) + 8 + 3) / 4 * 4;
constexpr size_t kOffQpad = 0;
constexpr size_t kOffEnv = kOffQpad + align256(4 * kLqMax * sizeof(float));
constexpr size_t kOffZq = kOffEnv + align256((size_t)CDTW_NOALLOC_MAX_QUERY * sizeof(float2));
constexpr size_t kOffZq64 = kOffZq + align256((size_t)CDTW_NOALLOC_MAX_QUERY * sizeof(float));
constexpr size_t kOffMu = kOffZq64 + align256((size_t)CDTW_NOALLOC_MAX_QUERY * sizeof(double));
constexpr size_t kOffSigma = kOffMu + align256((size_t)CDTW_NOALLOC_MAX_WINDOWS * sizeof(double));
constexpr size_t kScratchEnd = kOffSigma + align256((size_t)CDTW_NOALLOC_MAX_WINDOWS * sizeof(float));
static_assert(kScratchEnd <= (size_t)CDTW_NOALLOC_SCRATCH_BYTES, "scratch layout exceeds its array");

static __device__ __align__(256) unsigned char noalloc_scratch[CDTW_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 128;
std::mutex g_setup_mu;
unsigned char* g_scratch_addr[kMaxDevices] = {nullptr};
unsigned long long g_scratch_ctx[kMaxDevices] = {0};  // context ID the address belongs to

// Driver entry points for the current context's unique ID, resolved through
// the runtime (the library does not link libcuda itself).
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);
CtxGetCurrentFn g_ctx_current = nullptr;
CtxGetIdFn g_ctx_id = nullptr;
bool g_ctx_fns_tried = false;

// Unique ID of the calling thread's current context; 0 when there is none yet
// (the runtime creates the primary context on its first real call) or the
// driver cannot tell.
unsigned long long current_context_id() {
    if (!g_ctx_fns_tried) {
        g_ctx_fns_tried = true;
        void* f1 = nullptr;
        void* f2 = nullptr;
        cudaDriverEntryPointQueryResult r1, r2;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &r1) ==
                cudaSuccess &&
            r1 == cudaDriverEntryPointSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &r2) == cudaSuccess &&
            r2 == cudaDriverEntryPointSuccess) {
            g_ctx_current = (CtxGetCurrentFn)f1;
            g_ctx_id = (CtxGetIdFn)f2;
        }
        cudaGetLastError();
    }
    if (!g_ctx_current || !g_ctx_id) return 0;
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (g_ctx_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
    if (g_ctx_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Device address of the array on the current device: looked up once per
// device and context (cudaGetSymbolAddress with the device current), reused
// while the context stays the same.
cudaError_t scratch_address(int dev, unsigned char** out) {
    std::lock_guard<std::mutex> lock(g_setup_mu);
    const unsigned long long ctx = current_context_id();
    if (!g_scratch_addr[dev] || ctx == 0 || ctx != g_scratch_ctx[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr[dev] = (unsigned char*)p;
        // the lookup made the context current if there was none before
        g_scratch_ctx[dev] = ctx != 0 ? ctx : current_context_id();
    }
    *out = g_scratch_addr[dev];
    return cudaSuccess;
}

int fail(char* errbuf, int errlen, int status, const char* msg) {
    if (errbuf && errlen > 0) snprintf(errbuf, (size_t)errlen, "%s", msg);
    return status;
}

}  // namespace

extern "C" int cdtw_all_windows_noalloc(const float* d_query, int M, const float* d_subject,
                                        int64_t N, int W, int metric, float* d_out,
                                        void* cuda_stream, char* errbuf, int errlen) {
    using namespace cdtw;
    char msg[256];
    if (errbuf && errlen > 0) errbuf[0] = '\0';
    if (!d_query || !d_subject || !d_out)
        return fail(errbuf, errlen, CDTW_EINVAL, "null pointer");
    if (metric != CDTW_EUCLIDEAN && metric != CDTW_MANHATTAN)
        return fail(errbuf, errlen, CDTW_EINVAL, "metric must be CDTW_EUCLIDEAN or CDTW_MANHATTAN");
    if (M < 1 || N < M || W < 0)
        return fail(errbuf, errlen, CDTW_EINVAL, "need 1 <= M <= N and W >= 0");
    if (M > CDTW_NOALLOC_MAX_QUERY) {
        snprintf(msg, sizeof(msg), "query length %d exceeds the fixed-scratch limit %d", M,
                 CDTW_NOALLOC_MAX_QUERY);
        return fail(errbuf, errlen, CDTW_EUNSUPPORTED, msg);
    }
    const int64_t Nw = N - M + 1;
    if (Nw > CDTW_NOALLOC_MAX_WINDOWS) {
        snprintf(msg, sizeof(msg), "%lld windows exceed the fixed-scratch limit %d",
                 (long long)Nw, CDTW_NOALLOC_MAX_WINDOWS);
        return fail(errbuf, errlen, CDTW_EUNSUPPORTED, msg);
    }
    if (W > M - 1) W = M - 1;
    if (W > kNoAllocMaxBand) {
        snprintf(msg, sizeof(msg), "band %d exceeds the limit %d of this entry point", W,
                 kNoAllocMaxBand);
        return fail(errbuf, errlen, CDTW_EUNSUPPORTED, msg);
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return fail(errbuf, errlen, CDTW_ECUDA, "no current CUDA device");
    unsigned char* base = nullptr;
    e = scratch_address(dev, &base);
    if (e != cudaSuccess) {
        snprintf(msg, sizeof(msg), "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        return fail(errbuf, errlen, CDTW_ECUDA, msg);
    }
    // A handle-shaped record on the stack carries the stream and the query
    // pack into the shared launchers; it owns nothing and frees nothing.
    cdtw_handle_s rec;
    rec.device = dev;
    rec.stream = (cudaStream_t)cuda_stream;
    rec.q.M = M;
    rec.q.W = W;
    rec.q.lq = (int)((M + 2 * W + 8 + 3) / 4 * 4);
    rec.q.qpad = (float*)(base + kOffQpad);
    rec.q.env = (float2*)(base + kOffEnv);
    rec.q.zq = (float*)(base + kOffZq);
    rec.q.zq64 = (double*)(base + kOffZq64);
    rec.has_query = true;
    double* mu = (double*)(base + kOffMu);
    float* sigma = (float*)(base + kOffSigma);
    // Every region read below is fully written first in stream order, so
    // nothing in the array needs clearing between calls.
    int st = launch_prepare_query(&rec, d_query, M, W);
    if (st == CDTW_OK) st = launch_avg_std(&rec, d_subject, N, M, mu, sigma);
    if (st == CDTW_OK)
        st = launch_cdtw_windows(&rec, d_subject, N, mu, sigma, nullptr, Nw,
                                 metric == CDTW_EUCLIDEAN, d_out);
    if (st != CDTW_OK) return fail(errbuf, errlen, st, rec.err);
    return CDTW_OK;
}
