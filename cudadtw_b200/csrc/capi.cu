// C ABI entry points (include/cudadtw.h): handle lifecycle, argument checks,
// workspace management, and the host-buffer convenience calls.
#include "common.cuh"

#include <new>

namespace cdtw {

int set_error(cdtw_handle h, int status, const char* fmt, ...) {
    if (h) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(h->err, sizeof(h->err), fmt, ap);
        va_end(ap);
    }
    return status;
}

int check_cuda(cdtw_handle h, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return CDTW_OK;
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        return set_error(h, CDTW_ENOMEM, "%s: %s", what, cudaGetErrorString(e));
    }
    return set_error(h, CDTW_ECUDA, "%s: %s", what, cudaGetErrorString(e));
}

int check_memory_limit(cdtw_handle h, size_t freed, size_t bytes, const char* what) {
    if (h->mem_limit == 0) return CDTW_OK;
    const size_t held =
        h->ws_bytes + h->qmem_bytes + h->ring_bytes + h->batch_bytes + h->stream_bytes;
    if (held - std::min(held, freed) + bytes <= h->mem_limit) return CDTW_OK;
    return set_error(h, CDTW_ENOMEM,
                     "%s needs %zu bytes of device memory: above the handle's limit of %zu "
                     "(holding %zu)",
                     what, bytes, h->mem_limit, held);
}

int ensure_workspace(cdtw_handle h, size_t bytes) {
    if (bytes <= h->ws_bytes) return CDTW_OK;
    CDTW_TRY(check_memory_limit(h, h->ws_bytes, round_up((int64_t)bytes, 1 << 20),
                                "work area"));
    if (h->ws) {
        // the old block may still be in use by queued work on the stream
        CDTW_CUDA(h, cudaStreamSynchronize(h->stream));
        CDTW_CUDA(h, cudaFree(h->ws));
        h->ws = nullptr;
        h->ws_bytes = 0;
    }
    const size_t want = round_up((int64_t)bytes, 1 << 20);
    CDTW_CUDA(h, cudaMalloc(&h->ws, want));
    h->ws_bytes = want;
    return CDTW_OK;
}

// Sub-allocation of the workspace: 256-byte aligned slices.
struct Carver {
    size_t off = 0;
    template <class T>
    size_t take(size_t count) {
        const size_t o = off;
        off = (size_t)round_up((int64_t)(off + count * sizeof(T)), 256);
        return o;
    }
};

}  // namespace cdtw

size_t cdtw::query_pack_layout(int M, int W, QueryPack* q, char* base) {
    const int lq = qpad_len(M, W);
    Carver c;
    const size_t o_qpad = c.take<float>(4 * (size_t)lq);
    const size_t o_env = c.take<float2>(M);
    const size_t o_zq = c.take<float>(M);
    const size_t o_zq64 = c.take<double>(M);
    const int lqr = qrev_len(M, W);
    const size_t o_qrev = c.take<float>(4 * (size_t)lqr);
    const size_t o_qraw = c.take<float>(M);
    if (q && base) {
        q->M = M;
        q->W = W;
        q->lq = lq;
        q->qpad = (float*)(base + o_qpad);
        q->env = (float2*)(base + o_env);
        q->zq = (float*)(base + o_zq);
        q->zq64 = (double*)(base + o_zq64);
        q->lqr = lqr;
        q->qrev_base = qrev_hi(M, W);
        q->qrev = (float*)(base + o_qrev);
        q->qraw = (float*)(base + o_qraw);
    }
    return c.off;
}

namespace cdtw {

static int ensure_query_mem(cdtw_handle h, int M, int W) {
    const size_t bytes = query_pack_layout(M, W, nullptr, nullptr);
    if (bytes > h->qmem_bytes) {
        CDTW_TRY(check_memory_limit(h, h->qmem_bytes, bytes, "query pack"));
        if (h->qmem) {
            CDTW_CUDA(h, cudaStreamSynchronize(h->stream));
            CDTW_CUDA(h, cudaFree(h->qmem));
            h->qmem = nullptr;
            h->qmem_bytes = 0;
        }
        CDTW_CUDA(h, cudaMalloc(&h->qmem, bytes));
        h->qmem_bytes = bytes;
    }
    query_pack_layout(M, W, &h->q, (char*)h->qmem);
    return CDTW_OK;
}

static bool valid_metric(int metric) { return metric == CDTW_EUCLIDEAN || metric == CDTW_MANHATTAN; }

// Reads the search result key and stage counts back (the one host sync).
static int finish_search(cdtw_handle h, const unsigned long long* key, const int* ctr, int64_t Nw,
                         bool euclid, int64_t* location, float* distance) {
    char* pin = (char*)h->pinned;
    CDTW_CUDA(h, cudaMemcpyAsync(pin, key, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                 h->stream));
    CDTW_CUDA(h, cudaMemcpyAsync(pin + 8, ctr, sizeof(int) * 6, cudaMemcpyDeviceToHost,
                                 h->stream));
    CDTW_CUDA(h, cudaStreamSynchronize(h->stream));
    unsigned long long k;
    int c[6];
    memcpy(&k, pin, 8);
    memcpy(c, pin + 8, sizeof(c));
    h->last_counts[0] = Nw;
    h->last_counts[1] = c[0];
    h->last_counts[2] = c[1];
    // the reference's termination flag: best < largest LB_Kim (ctr[5] holds
    // its bits; both are >= 0)
    h->last_flag = (uint32_t)(k >> 32) < (uint32_t)c[5] ? 1 : 0;
    if (k == ~0ull)
        return set_error(h, CDTW_EINVAL,
                         "no window has a finite distance (NaN or Inf in the query or in every "
                         "window of the subject)");
    if ((uint32_t)k == 0xffffffffu)  // only the seeds' upper bound: no window beat it
        return set_error(h, CDTW_ECUDA, "search kept the seed bound, not a window");
    const uint32_t bits = (uint32_t)(k >> 32);
    float d;
    memcpy(&d, &bits, 4);
    if (location) *location = (int64_t)(uint32_t)k;
    if (distance) *distance = euclid ? sqrtf(d) : d;
    return CDTW_OK;
}

}  // namespace cdtw

using namespace cdtw;

extern "C" {

int cdtw_create(cdtw_handle* out, int device) {
    if (!out) return CDTW_EINVAL;
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return CDTW_ECUDA;
    }
    if (device < 0 || device >= ndev) return CDTW_EINVAL;
    cdtw_handle h = new (std::nothrow) cdtw_handle_s();
    if (!h) return CDTW_ENOMEM;
    h->device = device;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, device) !=
            cudaSuccess ||
        cudaMallocHost(&h->pinned, 4096) != cudaSuccess) {
        cudaGetLastError();
        if (h->own_stream) cudaStreamDestroy(h->own_stream);
        delete h;
        return CDTW_ECUDA;
    }
    h->stream = h->own_stream;
    *out = h;
    return CDTW_OK;
}

int cdtw_destroy(cdtw_handle h) {
    if (!h) return CDTW_EINVAL;
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->stream);
    if (h->own_stream) cudaStreamSynchronize(h->own_stream);
    batch_plan_release(h);
    batch_pipe_release(h);
    stream_release(h);
    if (h->ws) cudaFree(h->ws);
    if (h->qmem) cudaFree(h->qmem);
    if (h->ring) cudaFree(h->ring);
    if (h->pinned) cudaFreeHost(h->pinned);
    if (h->own_stream) cudaStreamDestroy(h->own_stream);
    if (h->xready) {
        for (cudaStream_t st : h->xfer) cudaStreamDestroy(st);
        for (cudaEvent_t ev : h->xev) cudaEventDestroy(ev);
    }
    delete h;
    return CDTW_OK;
}

int cdtw_set_stream(cdtw_handle h, void* cuda_stream) {
    if (!h) return CDTW_EINVAL;
    h->stream = (cudaStream_t)cuda_stream;  // NULL is the legacy default stream
    return CDTW_OK;
}

const char* cdtw_last_error(cdtw_handle h) { return h ? h->err : "null handle"; }

const char* cdtw_status_string(int status) {
    switch (status) {
        case CDTW_OK: return "ok";
        case CDTW_EINVAL: return "invalid argument";
        case CDTW_ENOMEM: return "out of memory";
        case CDTW_ECUDA: return "CUDA error";
        case CDTW_ETIMEOUT: return "device wait timed out";
        case CDTW_EUNSUPPORTED: return "unsupported";
        default: return "unknown status";
    }
}

int cdtw_band_from_percent(int M, int P) { return (int)(M * (P * 0.01)); }

int cdtw_avg_std(cdtw_handle h, const float* d_series, int64_t N, int M, double* d_avg,
                 float* d_std) {
    if (!h) return CDTW_EINVAL;
    if (!d_series || !d_avg || !d_std) return set_error(h, CDTW_EINVAL, "null pointer");
    if (M < 1 || N < M) return set_error(h, CDTW_EINVAL, "need 1 <= M <= N (M=%d N=%lld)", M,
                                         (long long)N);
    if (N - M + 1 > INT32_MAX) return set_error(h, CDTW_EUNSUPPORTED, "too many windows");
    CDTW_CUDA(h, cudaSetDevice(h->device));
    return launch_avg_std(h, d_series, N, M, d_avg, d_std);
}

int cdtw_set_query(cdtw_handle h, const float* query, int M, int W, int query_loc) {
    if (!h) return CDTW_EINVAL;
    if (!query) return set_error(h, CDTW_EINVAL, "null query");
    if (M < 1 || M > CDTW_MAX_QUERY)
        return set_error(h, CDTW_EINVAL, "query length %d outside [1, %d]", M, CDTW_MAX_QUERY);
    if (W < 0) return set_error(h, CDTW_EINVAL, "negative band %d", W);
    if (query_loc != CDTW_HOST && query_loc != CDTW_DEVICE)
        return set_error(h, CDTW_EINVAL, "bad query location %d", query_loc);
    if (W > M - 1) W = M - 1;  // a wider band changes nothing
    CDTW_CUDA(h, cudaSetDevice(h->device));
    CDTW_TRY(ensure_query_mem(h, M, W));
    const float* dq = query;
    if (query_loc == CDTW_HOST) {
        // stage the raw query in the (now unused) zq slot of the pack
        CDTW_CUDA(h, cudaMemcpyAsync(h->q.zq, query, sizeof(float) * M, cudaMemcpyHostToDevice,
                                     h->stream));
        dq = h->q.zq;
    }
    CDTW_TRY(launch_prepare_query(h, dq, M, W));
    h->has_query = true;
    return CDTW_OK;
}

int cdtw_gpu_cdtw(cdtw_handle h, const float* d_subject, int64_t N, const double* d_avg,
                  const float* d_std, const int32_t* d_indices, int64_t L, int metric,
                  float* d_out) {
    if (!h) return CDTW_EINVAL;
    if (!h->has_query) return set_error(h, CDTW_EINVAL, "no query set (cdtw_set_query)");
    if (!d_subject || !d_avg || !d_std || !d_out)
        return set_error(h, CDTW_EINVAL, "null pointer");
    if (!valid_metric(metric)) return set_error(h, CDTW_EINVAL, "bad metric %d", metric);
    const int M = h->q.M;
    if (N < M) return set_error(h, CDTW_EINVAL, "subject shorter than query");
    const int64_t Nw = N - M + 1;
    if (!d_indices) L = Nw;
    if (L < 0 || L > INT32_MAX) return set_error(h, CDTW_EINVAL, "bad index count");
    CDTW_CUDA(h, cudaSetDevice(h->device));
    return launch_cdtw_windows(h, d_subject, N, d_avg, d_std, d_indices, L,
                               metric == CDTW_EUCLIDEAN, d_out);
}

int cdtw_all_windows_host(cdtw_handle h, const float* h_query, int M, const float* h_subject,
                          int64_t N, int W, int metric, float* h_out) {
    if (!h) return CDTW_EINVAL;
    if (!h_query || !h_subject || !h_out) return set_error(h, CDTW_EINVAL, "null pointer");
    if (!valid_metric(metric)) return set_error(h, CDTW_EINVAL, "bad metric %d", metric);
    if (M < 1 || N < M) return set_error(h, CDTW_EINVAL, "need 1 <= M <= N");
    const int64_t Nw = N - M + 1;
    if (Nw > INT32_MAX) return set_error(h, CDTW_EUNSUPPORTED, "too many windows");
    CDTW_CUDA(h, cudaSetDevice(h->device));
    Carver c;
    const size_t o_x = c.take<float>(N);
    const size_t o_mu = c.take<double>(Nw);
    const size_t o_sd = c.take<float>(Nw);
    const size_t o_out = c.take<float>(Nw);
    CDTW_TRY(ensure_workspace(h, c.off));
    char* base = (char*)h->ws;
    float* dx = (float*)(base + o_x);
    double* dmu = (double*)(base + o_mu);
    float* dsd = (float*)(base + o_sd);
    float* dout = (float*)(base + o_out);
    CDTW_TRY(cdtw_set_query(h, h_query, M, W, CDTW_HOST));
    // pipeline over window chunks (multiples of the statistics kernel's
    // 2048-window warp runs, so per-chunk statistics equal the whole-stream
    // ones): samples in on xfer[0], statistics + cDTW alternately on the
    // handle's stream and xfer[2] (a chunk's first waves overlap the previous
    // chunk's last), results out on xfer[1]; copies overlap compute
    if (!h->xready) {
        for (cudaStream_t& st : h->xfer)
            CDTW_CUDA(h, cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        for (cudaEvent_t& ev : h->xev)
            CDTW_CUDA(h, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        h->xready = true;
    }
    const int64_t run = 2048;
    const int64_t chunk =
        round_up(std::max<int64_t>(div_up(Nw, 16), std::min<int64_t>(Nw, (int64_t)1 << 19)), run);
    const int nch = (int)div_up(Nw, chunk);
    cudaEvent_t start = h->xev[3 * 16];
    CDTW_CUDA(h, cudaEventRecord(start, h->stream));  // after earlier work on the workspace
    for (cudaStream_t st : h->xfer) CDTW_CUDA(h, cudaStreamWaitEvent(st, start, 0));
    const bool eu = metric == CDTW_EUCLIDEAN;
    cudaStream_t const user = h->stream;
    // strip kernels share the handle's ring buffer: their chunks stay on one stream
    const int variant = choose_variant(h, h->q.W);
    const bool alternate = variant == CDTW_VARIANT_REGISTER || variant == CDTW_VARIANT_LANE;
    cudaStream_t const comp[2] = {user, alternate ? h->xfer[2] : user};
    int64_t copied = 0;  // samples already on the device
    for (int i = 0; i < nch; ++i) {
        const int64_t c0 = (int64_t)i * chunk, c1 = std::min(Nw, c0 + chunk);
        const int64_t s1 = c1 + M - 1;  // samples chunk i needs: [c0, s1)
        cudaEvent_t in = h->xev[3 * i], done = h->xev[3 * i + 1];
        CDTW_CUDA(h, cudaMemcpyAsync(dx + copied, h_subject + copied,
                                     sizeof(float) * (s1 - copied), cudaMemcpyHostToDevice,
                                     h->xfer[0]));
        copied = s1;
        CDTW_CUDA(h, cudaEventRecord(in, h->xfer[0]));
        h->stream = comp[i & 1];
        int st = cudaStreamWaitEvent(h->stream, in, 0) == cudaSuccess ? CDTW_OK : CDTW_ECUDA;
        if (st == CDTW_OK) st = launch_avg_std(h, dx + c0, s1 - c0, M, dmu + c0, dsd + c0);
        if (st == CDTW_OK)
            st = launch_cdtw_windows(h, dx + c0, s1 - c0, dmu + c0, dsd + c0, nullptr, c1 - c0,
                                     eu, dout + c0);
        if (st == CDTW_OK && cudaEventRecord(done, h->stream) != cudaSuccess) st = CDTW_ECUDA;
        h->stream = user;
        if (st != CDTW_OK) return st == CDTW_ECUDA ? check_cuda(h, cudaGetLastError(), "pipeline") : st;
        CDTW_CUDA(h, cudaStreamWaitEvent(h->xfer[1], done, 0));
        CDTW_CUDA(h, cudaMemcpyAsync(h_out + c0, dout + c0, sizeof(float) * (c1 - c0),
                                     cudaMemcpyDeviceToHost, h->xfer[1]));
    }
    CDTW_CUDA(h, cudaStreamSynchronize(h->xfer[1]));
    CDTW_CUDA(h, cudaStreamSynchronize(h->xfer[2]));
    CDTW_CUDA(h, cudaStreamSynchronize(h->stream));
    return CDTW_OK;
}

int cdtw_lb_kim(cdtw_handle h, const float* d_subject, int64_t N, const double* d_avg,
                const float* d_std, const int32_t* d_indices, int64_t L, int metric,
                float* d_out) {
    if (!h) return CDTW_EINVAL;
    if (!h->has_query) return set_error(h, CDTW_EINVAL, "no query set (cdtw_set_query)");
    if (!d_subject || !d_avg || !d_std || !d_out) return set_error(h, CDTW_EINVAL, "null pointer");
    if (!valid_metric(metric)) return set_error(h, CDTW_EINVAL, "bad metric %d", metric);
    if (N < h->q.M) return set_error(h, CDTW_EINVAL, "subject shorter than query");
    if (!d_indices) L = N - h->q.M + 1;
    if (L < 0 || L > INT32_MAX) return set_error(h, CDTW_EINVAL, "bad index count");
    CDTW_CUDA(h, cudaSetDevice(h->device));
    return launch_lb_kim(h, d_subject, N, d_avg, d_std, d_indices, L, metric == CDTW_EUCLIDEAN,
                         d_out);
}

int cdtw_lb_keogh(cdtw_handle h, const float* d_subject, int64_t N, const double* d_avg,
                  const float* d_std, const int32_t* d_indices, int64_t L, int metric,
                  float* d_fwd, float* d_rev) {
    if (!h) return CDTW_EINVAL;
    if (!h->has_query) return set_error(h, CDTW_EINVAL, "no query set (cdtw_set_query)");
    if (!d_subject || !d_avg || !d_std || (!d_fwd && !d_rev))
        return set_error(h, CDTW_EINVAL, "null pointer");
    if (!valid_metric(metric)) return set_error(h, CDTW_EINVAL, "bad metric %d", metric);
    if (N < h->q.M) return set_error(h, CDTW_EINVAL, "subject shorter than query");
    if (!d_indices) L = N - h->q.M + 1;
    if (L < 0 || L > INT32_MAX) return set_error(h, CDTW_EINVAL, "bad index count");
    CDTW_CUDA(h, cudaSetDevice(h->device));
    float2* xenv = nullptr;
    if (d_rev) {
        Carver c;
        const size_t o_env = c.take<float2>(N);
        const size_t o_scr = c.take<char>(stream_envelope_scratch_bytes(N));
        CDTW_TRY(ensure_workspace(h, c.off));
        xenv = (float2*)((char*)h->ws + o_env);
        CDTW_TRY(launch_stream_envelope(h, d_subject, N, h->q.W, (float*)((char*)h->ws + o_scr),
                                        xenv));
    }
    return launch_lb_keogh(h, d_subject, N, d_avg, d_std, xenv, d_indices, L,
                           metric == CDTW_EUCLIDEAN, d_fwd, d_rev);
}

int cdtw_prune_cdtw(cdtw_handle h, const float* d_subject, int64_t N, const double* d_avg,
                    const float* d_std, int metric, int64_t* location, float* distance) {
    if (!h) return CDTW_EINVAL;
    if (!h->has_query) return set_error(h, CDTW_EINVAL, "no query set (cdtw_set_query)");
    if (!d_subject || !d_avg || !d_std) return set_error(h, CDTW_EINVAL, "null pointer");
    if (!valid_metric(metric)) return set_error(h, CDTW_EINVAL, "bad metric %d", metric);
    const int M = h->q.M;
    if (M < 11)
        return set_error(h, CDTW_EINVAL,
                         "the search's LB_Kim is a 10-point DTW: query length must be >= 11");
    if (N < M) return set_error(h, CDTW_EINVAL, "subject shorter than query");
    if (N - M + 1 > INT32_MAX) return set_error(h, CDTW_EUNSUPPORTED, "too many windows");
    CDTW_CUDA(h, cudaSetDevice(h->device));
    CDTW_TRY(ensure_workspace(h, search_workspace_bytes(N, M, h->q.W)));
    unsigned long long* key;
    int* ctr;
    CDTW_TRY(run_search(h, d_subject, N, d_avg, d_std, metric == CDTW_EUCLIDEAN, (char*)h->ws,
                        &key, &ctr));
    return finish_search(h, key, ctr, N - M + 1, metric == CDTW_EUCLIDEAN, location, distance);
}

int cdtw_topk(cdtw_handle h, const float* d_subject, int64_t N, const double* d_avg,
              const float* d_std, int metric, int k, int64_t* locations, float* distances,
              int* found) {
    if (!h) return CDTW_EINVAL;
    if (found) *found = 0;
    if (!h->has_query) return set_error(h, CDTW_EINVAL, "no query set (cdtw_set_query)");
    const int M = h->q.M;
    if (!d_subject || !d_avg || !d_std || !locations || k < 1)
        return set_error(h, CDTW_EINVAL, "bad top-k arguments");
    if (N < M || N - M + 1 > (int64_t)INT32_MAX)
        return set_error(h, CDTW_EINVAL, "subject length %lld for M=%d", (long long)N, M);
    if (M < 11) return set_error(h, CDTW_EUNSUPPORTED, "top-k search needs M >= 11");
    if (!valid_metric(metric)) return set_error(h, CDTW_EINVAL, "bad metric %d", metric);
    CDTW_CUDA(h, cudaSetDevice(h->device));
    CDTW_TRY(ensure_workspace(h, topk_workspace_bytes(N, M, h->q.W)));
    std::vector<unsigned long long> picks;
    CDTW_TRY(run_topk(h, d_subject, N, d_avg, d_std, metric == CDTW_EUCLIDEAN, k,
                      (char*)h->ws, &picks));
    for (size_t i = 0; i < picks.size(); ++i) {
        const uint32_t bits = (uint32_t)(picks[i] >> 32);
        float d;
        memcpy(&d, &bits, 4);
        locations[i] = (int64_t)(uint32_t)picks[i];
        if (distances) distances[i] = metric == CDTW_EUCLIDEAN ? sqrtf(d) : d;
    }
    if (found) *found = (int)picks.size();
    return CDTW_OK;
}

int cdtw_topk_device(cdtw_handle h, const float* d_subject, int64_t N, const double* d_avg,
                     const float* d_std, int metric, int k, int64_t* locations,
                     float* distances, int* found) {
    if (!h) return CDTW_EINVAL;
    if (found) *found = 0;
    if (!h->has_query) return set_error(h, CDTW_EINVAL, "no query set (cdtw_set_query)");
    const int M = h->q.M;
    if (!d_subject || !d_avg || !d_std || !locations || k < 1)
        return set_error(h, CDTW_EINVAL, "bad top-k arguments");
    if (N < M || N - M + 1 > (int64_t)INT32_MAX)
        return set_error(h, CDTW_EINVAL, "subject length %lld for M=%d", (long long)N, M);
    if (M < 11) return set_error(h, CDTW_EUNSUPPORTED, "top-k search needs M >= 11");
    if (!valid_metric(metric)) return set_error(h, CDTW_EINVAL, "bad metric %d", metric);
    if (k > (N - M + 1)) k = (int)(N - M + 1);
    CDTW_CUDA(h, cudaSetDevice(h->device));
    Carver c;
    const size_t o_ws = c.take<char>(topk_device_workspace_bytes(N, M, h->q.W, k));
    const size_t o_pk = c.take<int32_t>(k);
    const size_t o_pd = c.take<float>(k);
    const size_t o_n = c.take<int>(2);
    CDTW_TRY(ensure_workspace(h, c.off));
    char* base = (char*)h->ws;
    int32_t* picks = (int32_t*)(base + o_pk);
    float* pick_d = (float*)(base + o_pd);
    int* cnt = (int*)(base + o_n);
    CDTW_TRY(run_topk_device(h, d_subject, N, d_avg, d_std, metric == CDTW_EUCLIDEAN, k, k,
                             base + o_ws, nullptr, nullptr, picks, pick_d, cnt, cnt + 1));
    int hc[2];
    std::vector<int32_t> hp(k);
    std::vector<float> hd(k);
    CDTW_CUDA(h, cudaMemcpyAsync(hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, h->stream));
    CDTW_CUDA(h, cudaMemcpyAsync(hp.data(), picks, sizeof(int32_t) * k, cudaMemcpyDeviceToHost,
                                 h->stream));
    CDTW_CUDA(h, cudaMemcpyAsync(hd.data(), pick_d, sizeof(float) * k, cudaMemcpyDeviceToHost,
                                 h->stream));
    CDTW_CUDA(h, cudaStreamSynchronize(h->stream));
    if (hc[1] != 0)
        return set_error(h, CDTW_EUNSUPPORTED,
                         "more windows under the top-k threshold than the hit list holds");
    const int n = std::min(hc[0], k);
    for (int i = 0; i < n; ++i) {
        locations[i] = hp[i];
        if (distances) distances[i] = metric == CDTW_EUCLIDEAN ? sqrtf(hd[i]) : hd[i];
    }
    if (found) *found = n;
    return CDTW_OK;
}

int cdtw_search_host(cdtw_handle h, const float* h_query, int M, const float* h_subject,
                     int64_t N, int W, int metric, int64_t* location, float* distance) {
    if (!h) return CDTW_EINVAL;
    if (!h_query || !h_subject) return set_error(h, CDTW_EINVAL, "null pointer");
    if (!valid_metric(metric)) return set_error(h, CDTW_EINVAL, "bad metric %d", metric);
    if (M < 11) return set_error(h, CDTW_EINVAL, "query length must be >= 11 (LB_Kim)");
    if (N < M) return set_error(h, CDTW_EINVAL, "subject shorter than query");
    const int64_t Nw = N - M + 1;
    if (Nw > INT32_MAX) return set_error(h, CDTW_EUNSUPPORTED, "too many windows");
    CDTW_CUDA(h, cudaSetDevice(h->device));
    Carver c;
    const size_t o_x = c.take<float>(N);
    const size_t o_mu = c.take<double>(Nw);
    const size_t o_sd = c.take<float>(Nw);
    const size_t o_ws = c.take<char>(search_workspace_bytes(N, M, std::min(W, M - 1)));
    CDTW_TRY(ensure_workspace(h, c.off));
    char* base = (char*)h->ws;
    float* dx = (float*)(base + o_x);
    double* dmu = (double*)(base + o_mu);
    float* dsd = (float*)(base + o_sd);
    CDTW_CUDA(h, cudaMemcpyAsync(dx, h_subject, sizeof(float) * N, cudaMemcpyHostToDevice,
                                 h->stream));
    CDTW_TRY(cdtw_set_query(h, h_query, M, W, CDTW_HOST));
    CDTW_TRY(launch_avg_std(h, dx, N, M, dmu, dsd));
    unsigned long long* key;
    int* ctr;
    CDTW_TRY(run_search(h, dx, N, dmu, dsd, metric == CDTW_EUCLIDEAN, base + o_ws, &key, &ctr));
    return finish_search(h, key, ctr, Nw, metric == CDTW_EUCLIDEAN, location, distance);
}

// ---- GPU-ED -------------------------------------------------------------------

static int ed_run(cdtw_handle h, const double* dq, int M, const double* dx, int64_t N,
                  double* dout, char* base, size_t* used) {
    const int64_t Nw = N - M + 1;
    Carver c;
    c.off = *used;
    const size_t o_zq = c.take<double>(M);
    const size_t o_mu = c.take<double>(Nw);
    const size_t o_sd = c.take<double>(Nw);
    *used = c.off;
    if (!base) return CDTW_OK;
    double* zq = (double*)(base + o_zq);
    double* mu = (double*)(base + o_mu);
    double* sd = (double*)(base + o_sd);
    CDTW_TRY(launch_znorm64(h, dq, M, zq));
    CDTW_TRY(launch_avg_std64(h, dx, N, M, mu, sd));
    return launch_ed(h, dx, N, zq, M, sd, dout);
}

int ed_all_windows(cdtw_handle h, const double* d_query, int M, const double* d_subject,
                   int64_t N, double* d_out) {
    if (!h) return CDTW_EINVAL;
    if (!d_query || !d_subject || !d_out) return set_error(h, CDTW_EINVAL, "null pointer");
    if (M < 1 || M > CDTW_MAX_QUERY || N < M)
        return set_error(h, CDTW_EINVAL, "need 1 <= M <= min(N, %d)", CDTW_MAX_QUERY);
    CDTW_CUDA(h, cudaSetDevice(h->device));
    size_t used = 0;
    ed_run(h, d_query, M, d_subject, N, d_out, nullptr, &used);
    CDTW_TRY(ensure_workspace(h, used));
    used = 0;
    return ed_run(h, d_query, M, d_subject, N, d_out, (char*)h->ws, &used);
}

int ed_search_host(cdtw_handle h, const double* h_query, int M, const double* h_subject,
                   int64_t N, int64_t* location, double* distance) {
    if (!h) return CDTW_EINVAL;
    if (!h_query || !h_subject) return set_error(h, CDTW_EINVAL, "null pointer");
    if (M < 1 || M > CDTW_MAX_QUERY || N < M)
        return set_error(h, CDTW_EINVAL, "need 1 <= M <= min(N, %d)", CDTW_MAX_QUERY);
    CDTW_CUDA(h, cudaSetDevice(h->device));
    const int64_t Nw = N - M + 1;
    Carver c;
    const size_t o_q = c.take<double>(M);
    const size_t o_x = c.take<double>(N);
    const size_t o_d = c.take<double>(Nw);
    const size_t o_p = c.take<ArgMin64>(argmin64_partials(Nw));
    const size_t o_r = c.take<ArgMin64>(1);
    size_t used = c.off;
    ed_run(h, nullptr, M, nullptr, N, nullptr, nullptr, &used);
    CDTW_TRY(ensure_workspace(h, used));
    char* base = (char*)h->ws;
    CDTW_CUDA(h, cudaMemcpyAsync(base + o_q, h_query, sizeof(double) * M, cudaMemcpyHostToDevice,
                                 h->stream));
    CDTW_CUDA(h, cudaMemcpyAsync(base + o_x, h_subject, sizeof(double) * N,
                                 cudaMemcpyHostToDevice, h->stream));
    used = c.off;
    CDTW_TRY(ed_run(h, (double*)(base + o_q), M, (double*)(base + o_x), N,
                    (double*)(base + o_d), base, &used));
    CDTW_TRY(launch_argmin64(h, (double*)(base + o_d), Nw, (ArgMin64*)(base + o_p),
                             (ArgMin64*)(base + o_r)));
    ArgMin64* pin = (ArgMin64*)h->pinned;
    CDTW_CUDA(h, cudaMemcpyAsync(pin, base + o_r, sizeof(ArgMin64), cudaMemcpyDeviceToHost,
                                 h->stream));
    CDTW_CUDA(h, cudaStreamSynchronize(h->stream));
    if (location) *location = pin->i;
    if (distance) *distance = sqrt(fmax(pin->v, 0.0));
    return CDTW_OK;
}

// ---- GPU-LDTW -----------------------------------------------------------------

int ldtw_all_windows(cdtw_handle h, const float* d_subject, int64_t N, int metric,
                     double* d_out) {
    if (!h) return CDTW_EINVAL;
    if (!h->has_query) return set_error(h, CDTW_EINVAL, "no query set (cdtw_set_query)");
    if (!d_subject || !d_out) return set_error(h, CDTW_EINVAL, "null pointer");
    if (!valid_metric(metric)) return set_error(h, CDTW_EINVAL, "bad metric %d", metric);
    const int M = h->q.M;
    if (N < M) return set_error(h, CDTW_EINVAL, "subject shorter than query");
    CDTW_CUDA(h, cudaSetDevice(h->device));
    const int64_t Nw = N - M + 1;
    Carver c;
    const size_t o_mu = c.take<double>(Nw);
    const size_t o_sd = c.take<double>(Nw);
    CDTW_TRY(ensure_workspace(h, c.off));
    char* base = (char*)h->ws;
    CDTW_TRY(launch_avg_std64(h, d_subject, N, M, (double*)(base + o_mu), (double*)(base + o_sd)));
    return launch_ldtw(h, d_subject, N, (double*)(base + o_mu), (double*)(base + o_sd),
                       metric == CDTW_EUCLIDEAN, d_out);
}

int ldtw_search_host(cdtw_handle h, const float* h_query, int M, const float* h_subject,
                     int64_t N, int W, int metric, int64_t* location, double* distance) {
    if (!h) return CDTW_EINVAL;
    if (!h_query || !h_subject) return set_error(h, CDTW_EINVAL, "null pointer");
    if (!valid_metric(metric)) return set_error(h, CDTW_EINVAL, "bad metric %d", metric);
    if (M < 1 || N < M) return set_error(h, CDTW_EINVAL, "need 1 <= M <= N");
    CDTW_CUDA(h, cudaSetDevice(h->device));
    const int64_t Nw = N - M + 1;
    Carver c;
    const size_t o_x = c.take<float>(N);
    const size_t o_mu = c.take<double>(Nw);
    const size_t o_sd = c.take<double>(Nw);
    const size_t o_d = c.take<double>(Nw);
    const size_t o_p = c.take<ArgMin64>(argmin64_partials(Nw));
    const size_t o_r = c.take<ArgMin64>(1);
    CDTW_TRY(ensure_workspace(h, c.off));
    char* base = (char*)h->ws;
    float* dx = (float*)(base + o_x);
    CDTW_CUDA(h, cudaMemcpyAsync(dx, h_subject, sizeof(float) * N, cudaMemcpyHostToDevice,
                                 h->stream));
    CDTW_TRY(cdtw_set_query(h, h_query, M, W, CDTW_HOST));
    CDTW_TRY(launch_avg_std64(h, dx, N, M, (double*)(base + o_mu), (double*)(base + o_sd)));
    CDTW_TRY(launch_ldtw(h, dx, N, (double*)(base + o_mu), (double*)(base + o_sd),
                         metric == CDTW_EUCLIDEAN, (double*)(base + o_d)));
    CDTW_TRY(launch_argmin64(h, (double*)(base + o_d), Nw, (ArgMin64*)(base + o_p),
                             (ArgMin64*)(base + o_r)));
    ArgMin64* pin = (ArgMin64*)h->pinned;
    CDTW_CUDA(h, cudaMemcpyAsync(pin, base + o_r, sizeof(ArgMin64), cudaMemcpyDeviceToHost,
                                 h->stream));
    CDTW_CUDA(h, cudaStreamSynchronize(h->stream));
    if (location) *location = pin->i;
    if (distance) *distance = metric == CDTW_EUCLIDEAN ? sqrt(pin->v) : pin->v;
    return CDTW_OK;
}

int ldtw_ref_all_windows(cdtw_handle h, const float* d_subject, int64_t N, int metric, int znorm,
                         float* d_out) {
    if (!h) return CDTW_EINVAL;
    if (!h->has_query) return set_error(h, CDTW_EINVAL, "no query set (cdtw_set_query)");
    if (!d_subject || !d_out) return set_error(h, CDTW_EINVAL, "null pointer");
    if (!valid_metric(metric)) return set_error(h, CDTW_EINVAL, "bad metric %d", metric);
    const int M = h->q.M;
    if (N < M) return set_error(h, CDTW_EINVAL, "subject shorter than query");
    if (N - M + 1 > INT32_MAX) return set_error(h, CDTW_EUNSUPPORTED, "too many windows");
    CDTW_CUDA(h, cudaSetDevice(h->device));
    Carver c;
    const size_t o_q = c.take<float>(M);
    CDTW_TRY(ensure_workspace(h, c.off));
    return launch_ldtw_ref(h, d_subject, N, metric == CDTW_EUCLIDEAN, znorm != 0,
                           (float*)((char*)h->ws + o_q), d_out);
}

int ldtw_ref_search_host(cdtw_handle h, const float* h_query, int M, const float* h_subject,
                         int64_t N, int W, int metric, int znorm, int64_t* location,
                         float* distance) {
    if (!h) return CDTW_EINVAL;
    if (!h_query || !h_subject) return set_error(h, CDTW_EINVAL, "null pointer");
    if (!valid_metric(metric)) return set_error(h, CDTW_EINVAL, "bad metric %d", metric);
    if (M < 1 || N < M) return set_error(h, CDTW_EINVAL, "need 1 <= M <= N");
    const int64_t Nw = N - M + 1;
    if (Nw > INT32_MAX) return set_error(h, CDTW_EUNSUPPORTED, "too many windows");
    CDTW_CUDA(h, cudaSetDevice(h->device));
    Carver c;
    const size_t o_x = c.take<float>(N);
    const size_t o_q = c.take<float>(M);
    const size_t o_d = c.take<float>(Nw);
    const size_t o_k = c.take<unsigned long long>(1);
    CDTW_TRY(ensure_workspace(h, c.off));
    char* base = (char*)h->ws;
    float* dx = (float*)(base + o_x);
    CDTW_CUDA(h, cudaMemcpyAsync(dx, h_subject, sizeof(float) * N, cudaMemcpyHostToDevice,
                                 h->stream));
    CDTW_TRY(cdtw_set_query(h, h_query, M, W, CDTW_HOST));
    CDTW_TRY(launch_ldtw_ref(h, dx, N, metric == CDTW_EUCLIDEAN, znorm != 0,
                             (float*)(base + o_q), (float*)(base + o_d)));
    unsigned long long* key = (unsigned long long*)(base + o_k);
    CDTW_CUDA(h, cudaMemsetAsync(key, 0xff, sizeof(unsigned long long), h->stream));
    CDTW_TRY(launch_argmin_f32(h, (float*)(base + o_d), Nw, key));
    unsigned long long* pin = (unsigned long long*)h->pinned;
    CDTW_CUDA(h, cudaMemcpyAsync(pin, key, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                 h->stream));
    CDTW_CUDA(h, cudaStreamSynchronize(h->stream));
    if (*pin == ~0ull)
        return set_error(h, CDTW_EINVAL, "no window has a finite LDTW cost");
    const uint32_t bits = (uint32_t)(*pin >> 32);
    float d;
    memcpy(&d, &bits, 4);
    if (location) *location = (int64_t)(uint32_t)*pin;
    if (distance) *distance = metric == CDTW_EUCLIDEAN ? sqrtf(d) : d;
    return CDTW_OK;
}

size_t cdtw_pair_path_bytes(int64_t n, int L) {
    if (n <= 0 || L <= 0) return 0;
    return (size_t)n * 32 + (size_t)n * L * 8;
}

// Default cap on the direction scratch of one cdtw_pair_fwd call with a path
// record; above it (or above half the handle's memory limit) the forward
// recomputes from checkpoints instead.
static const size_t kPairDirBudget = (size_t)4 << 30;

// Path mode of a forward with a path record: true for the checkpointed
// recomputation, false for the stored direction bits.
static bool pair_recompute(size_t mem_limit, int64_t n, int L, int W, int flags) {
    if (pair_ckpt_floats(L, W) == 0) return false;  // shared-record pairs: no choice
    if (flags & CDTW_PAIR_RECOMPUTE) return true;
    if (flags & CDTW_PAIR_STORE_DIRS) return false;
    const size_t budget = mem_limit ? std::min(kPairDirBudget, mem_limit / 2) : kPairDirBudget;
    return (size_t)n * pair_dirs_words(L, W) * 4 > budget;
}

// Slices of the forward's work area: z copies, then the direction scratch or
// the checkpoints.
static size_t pair_carve(int64_t n, int L, int W, int flags, bool with_path, bool recompute,
                         size_t* o_zq, size_t* o_zs, size_t* o_path) {
    Carver c;
    const bool zn = flags & CDTW_PAIR_ZNORM;
    *o_zq = zn ? c.take<float>((size_t)n * L) : 0;
    *o_zs = zn ? c.take<float>((size_t)n * L) : 0;
    *o_path = 0;
    if (with_path)
        *o_path = recompute ? c.take<float>((size_t)n * pair_ckpt_floats(L, W))
                            : c.take<uint32_t>((size_t)n * pair_dirs_words(L, W));
    return c.off;
}

size_t cdtw_pair_workspace_bytes(int64_t n, int L, int W, int flags, int with_path) {
    if (n <= 0 || L < 1 || L > CDTW_MAX_QUERY || W < 0) return 0;
    W = std::min(W, L - 1);
    if (W > CDTW_PAIR_MAX_BAND) return 0;
    size_t a, b, c;
    return pair_carve(n, L, W, flags, with_path != 0, with_path && pair_recompute(0, n, L, W, flags),
                      &a, &b, &c);
}

static int pair_check(cdtw_handle h, const float* q, const float* s, int64_t n, int L,
                      int metric, int flags) {
    if (!q || !s || n < 0 || L < 1 || L > CDTW_MAX_QUERY)
        return set_error(h, CDTW_EINVAL, "bad pair arguments (n=%lld L=%d)", (long long)n, L);
    if (!valid_metric(metric)) return set_error(h, CDTW_EINVAL, "bad metric %d", metric);
    if (flags & ~(CDTW_PAIR_ZNORM | CDTW_PAIR_STORE_DIRS | CDTW_PAIR_RECOMPUTE))
        return set_error(h, CDTW_EINVAL, "bad flags %d", flags);
    if ((flags & CDTW_PAIR_STORE_DIRS) && (flags & CDTW_PAIR_RECOMPUTE))
        return set_error(h, CDTW_EINVAL, "CDTW_PAIR_STORE_DIRS and CDTW_PAIR_RECOMPUTE exclude "
                                         "each other");
    if (n > (int64_t)INT32_MAX * 4) return set_error(h, CDTW_EINVAL, "too many pairs");
    return CDTW_OK;
}

int cdtw_pair_fwd(cdtw_handle h, const float* d_q, const float* d_s, int64_t n, int L, int W,
                  int metric, int flags, float* d_D, void* d_path) {
    if (!h) return CDTW_EINVAL;
    CDTW_TRY(pair_check(h, d_q, d_s, n, L, metric, flags));
    if (!d_D || W < 0) return set_error(h, CDTW_EINVAL, "bad output or band");
    if (n == 0) return CDTW_OK;
    W = std::min(W, L - 1);
    if (W > CDTW_PAIR_MAX_BAND)
        return set_error(h, CDTW_EUNSUPPORTED, "pair band W=%d exceeds %d", W, CDTW_PAIR_MAX_BAND);
    if (d_path && ((uintptr_t)d_path & 7))
        return set_error(h, CDTW_EINVAL, "path record must be 8-byte aligned");
    const bool zn = flags & CDTW_PAIR_ZNORM;
    const bool recompute = d_path && pair_recompute(h->mem_limit, n, L, W, flags);
    size_t o_zq, o_zs, o_dirs;
    CDTW_TRY(ensure_workspace(
        h, pair_carve(n, L, W, flags, d_path != nullptr, recompute, &o_zq, &o_zs, &o_dirs)));
    h->last_pair_recompute = recompute ? 1 : 0;
    char* ws = (char*)h->ws;
    double* hdr = (double*)d_path;
    uint32_t* rows = d_path ? (uint32_t*)((char*)d_path + (size_t)n * 32) : nullptr;
    uint32_t* cols = d_path ? rows + (size_t)n * L : nullptr;
    const float* zq = d_q;
    const float* zs = d_s;
    if (zn) {
        CDTW_TRY(launch_pair_znorm(h, d_q, d_s, n, L, (float*)(ws + o_zq), (float*)(ws + o_zs),
                                   hdr));
        zq = (const float*)(ws + o_zq);
        zs = (const float*)(ws + o_zs);
    }
    if (recompute)
        return launch_pair_fwd_ckpt(h, zq, zs, n, L, W, metric == CDTW_EUCLIDEAN, d_D,
                                    (float*)(ws + o_dirs), rows, cols);
    return launch_pair_fwd(h, zq, zs, n, L, W, metric == CDTW_EUCLIDEAN, d_D,
                           d_path ? (uint32_t*)(ws + o_dirs) : nullptr, rows, cols);
}

int cdtw_pair_last_mode(cdtw_handle h, int* recompute) {
    if (!h || !recompute) return CDTW_EINVAL;
    *recompute = h->last_pair_recompute;
    return CDTW_OK;
}

int cdtw_pair_bwd(cdtw_handle h, const float* d_q, const float* d_s, int64_t n, int L,
                  int metric, int flags, const void* d_path, const float* d_dD, float* d_dq,
                  float* d_ds) {
    if (!h) return CDTW_EINVAL;
    CDTW_TRY(pair_check(h, d_q, d_s, n, L, metric, flags));
    if (!d_path) return set_error(h, CDTW_EINVAL, "no path record");
    if ((uintptr_t)d_path & 7) return set_error(h, CDTW_EINVAL, "path record must be 8-byte aligned");
    if (n == 0 || (!d_dq && !d_ds)) return CDTW_OK;
    const double* hdr = (flags & CDTW_PAIR_ZNORM) ? (const double*)d_path : nullptr;
    const uint32_t* rows = (const uint32_t*)((const char*)d_path + (size_t)n * 32);
    const uint32_t* cols = rows + (size_t)n * L;
    return launch_pair_bwd(h, d_q, d_s, n, L, hdr, rows, cols, d_dD, metric == CDTW_EUCLIDEAN,
                           d_dq, d_ds);
}

int cdtw_set_band_variant(cdtw_handle h, int w_lo, int w_hi, int variant) {
    if (!h) return CDTW_EINVAL;
    if (variant < CDTW_VARIANT_AUTO || variant > CDTW_VARIANT_LANE || w_lo < 0 || w_hi < w_lo)
        return set_error(h, CDTW_EINVAL, "bad band range or variant");
    for (int w = w_lo; w <= w_hi && w < CDTW_MAX_QUERY; ++w) h->band_variant[w] = (unsigned char)variant;
    return CDTW_OK;
}

int cdtw_set_memory_limit(cdtw_handle h, size_t bytes) {
    if (!h) return CDTW_EINVAL;
    h->mem_limit = bytes;
    return CDTW_OK;
}

int cdtw_search_flag(cdtw_handle h, int* flag) {
    if (!h || !flag) return CDTW_EINVAL;
    *flag = h->last_flag;
    return CDTW_OK;
}

int cdtw_search_counts(cdtw_handle h, int64_t* counts) {
    if (!h || !counts) return CDTW_EINVAL;
    for (int i = 0; i < 3; ++i) counts[i] = h->last_counts[i];
    return CDTW_OK;
}

}  // extern "C"
