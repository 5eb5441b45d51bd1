// Search over a stream that arrives in pieces (cdtw_stream_begin / push /
// end): the subject is never held whole on the device.
//
// Reference: avg_std splits the window statistics into epochs of 1e7 samples
// (include/stats.cuh:115-142) and UCR_DTW_BIN.cpp:579-707 reads the data in
// EPOCH-sized chunks, carrying the last m-1 samples into the next chunk and
// the best-so-far across chunks.  Here the samples the caller pushes are
// copied on a copy stream straight into the current device chunk (directly
// from page-locked memory, else through two pinned staging buffers); when C
// samples are in, the M-1 samples before them (the halo) are copied from the
// previous chunk's device buffer and the chunk's windows are searched on the
// handle's stream starting from the best distance of the earlier chunks (a
// device-side carried key: no host round trip between chunks).  Two device
// buffers alternate, so the copies into one chunk overlap the search of the
// previous one.  Windows are numbered globally: chunk k's
// windows start at k*C - (M-1) (chunk 0's at 0); ties keep the earliest.
// The buffers outlive a stream and serve the next one when large enough.
#include "common.cuh"

#include <algorithm>
#include <new>

namespace cdtw {

namespace {

constexpr int64_t kStreamChunkDefault = (int64_t)1 << 23;  // samples per chunk

// Running result on the device.
struct StreamBest {
    unsigned long long carried;  // (best distance bits, 0): the bound the next chunk starts from
    long long loc;               // global window of the best distance
    long long n1, n2;            // summed stage counts (after LB_Kim, reaching cDTW)
    unsigned kmax;               // largest LB_Kim of any window (float bits)
};

struct StreamState {
    int M = 0, W = 0, metric = 0;
    int64_t C = 0;           // samples per chunk
    float* stage[2] = {nullptr, nullptr};  // pinned staging, C floats each
    float* dbuf[2] = {nullptr, nullptr};   // device chunks, M-1 + C floats each
    double* mu = nullptr;    // window statistics of one chunk
    float* sigma = nullptr;
    char* sws = nullptr;     // search workspace of one chunk
    StreamBest* best = nullptr;
    void* dmem = nullptr;    // one device allocation for all of the above
    size_t dbytes = 0;       // its size
    int64_t scap = 0;        // floats per staging buffer
    cudaStream_t copy = nullptr;
    cudaEvent_t staged[2] = {nullptr, nullptr};  // H2D from stage[b] done
    cudaEvent_t pushed = nullptr;                // a push's copies from page-locked memory
    int slot = 0;                                // next staging buffer
    bool slot_used[2] = {false, false};
    cudaEvent_t done[2] = {nullptr, nullptr};    // search over dbuf[b] done
    cudaEvent_t copied[2] = {nullptr, nullptr};  // dbuf[b] filled (halo + chunk)
    bool active = false;     // between begin and end
    int64_t fill = 0;        // samples in the current staging buffer
    int64_t chunks = 0;      // chunks launched
    int64_t total = 0;       // samples pushed
    int cur = 0;             // current staging / device buffer
    bool used[2] = {false, false};

    // Ends a stream; the buffers, events and copy stream stay for the next.
    void finish() {
        active = false;
        fill = chunks = total = 0;
        cur = 0;
        used[0] = used[1] = false;
        slot = 0;
        slot_used[0] = slot_used[1] = false;
    }
    void free_stage() {
        for (int b = 0; b < 2; ++b) {
            if (stage[b]) cudaFreeHost(stage[b]);
            stage[b] = nullptr;
        }
        scap = 0;
    }
    void release() {
        if (copy) cudaStreamSynchronize(copy);
        free_stage();
        for (int b = 0; b < 2; ++b) {
            if (staged[b]) cudaEventDestroy(staged[b]);
            if (done[b]) cudaEventDestroy(done[b]);
            if (copied[b]) cudaEventDestroy(copied[b]);
        }
        if (pushed) cudaEventDestroy(pushed);
        if (dmem) cudaFree(dmem);
        if (copy) cudaStreamDestroy(copy);
        *this = StreamState();
    }
};

__global__ void stream_init_kernel(StreamBest* b) {
    b->carried = ~0ull;
    b->loc = -1;
    b->n1 = 0;
    b->n2 = 0;
    b->kmax = 0;
}

// After a chunk's search: a key below the carried bound (and naming a
// window) is the new best; the carried bound becomes (its distance, 0), so a
// later window of equal distance never replaces it.
__global__ void stream_merge_kernel(const unsigned long long* __restrict__ key,
                                    const int* __restrict__ ctr, long long base,
                                    StreamBest* __restrict__ b) {
    const unsigned long long k = *key;
    if (k < b->carried && (uint32_t)k != 0xffffffffu) {
        b->carried = k & 0xffffffff00000000ull;
        b->loc = base + (long long)(uint32_t)k;
    }
    b->n1 += ctr[0];
    b->n2 += ctr[1];
    b->kmax = max(b->kmax, (unsigned)ctr[5]);
}

StreamState* state(cdtw_handle h) { return reinterpret_cast<StreamState*>(h->stream_state); }

// Page-locked host memory can be copied to the device directly.
bool page_locked(const void* p) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();  // plain pageable memory on older drivers
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}

// Searches the chunk in device buffer `cur`, whose n new samples the pushes
// have already copied after the halo position: first the halo, the last M-1
// samples of the previous chunk (at [C, C+M-1) of its buffer), then the
// chunk's windows.
int launch_chunk(cdtw_handle h, StreamState& s, int64_t n) {
    const int b = s.cur, o = b ^ 1;
    const int M = s.M;
    float* d = s.dbuf[b];
    if (s.chunks > 0)  // after the previous chunk's copies (the same copy stream)
        CDTW_CUDA(h, cudaMemcpyAsync(d, s.dbuf[o] + s.C, sizeof(float) * (M - 1),
                                     cudaMemcpyDeviceToDevice, s.copy));
    CDTW_CUDA(h, cudaEventRecord(s.copied[b], s.copy));
    s.used[b] = true;
    // search: chunk 0 has no halo; later chunks start M-1 samples early
    const float* x = s.chunks == 0 ? d + (M - 1) : d;
    const int64_t N = s.chunks == 0 ? n : n + M - 1;
    const long long base = s.chunks == 0 ? 0 : (long long)(s.chunks * s.C - (M - 1));
    s.chunks += 1;
    if (N < M) return CDTW_OK;  // fewer than M samples so far: no window yet
    CDTW_CUDA(h, cudaStreamWaitEvent(h->stream, s.copied[b], 0));
    CDTW_TRY(launch_avg_std(h, x, N, M, s.mu, s.sigma));
    unsigned long long* key;
    int* ctr;
    CDTW_TRY(run_search(h, x, N, s.mu, s.sigma, s.metric == CDTW_EUCLIDEAN, s.sws, &key, &ctr,
                        &s.best->carried));
    stream_merge_kernel<<<1, 1, 0, h->stream>>>(key, ctr, base, s.best);
    CDTW_LAUNCH(h, "stream_merge_kernel");
    CDTW_CUDA(h, cudaEventRecord(s.done[b], h->stream));
    return CDTW_OK;
}

}  // namespace

void stream_release(cdtw_handle h) {
    StreamState* s = state(h);
    if (s) {
        s->release();
        delete s;
        h->stream_state = nullptr;
    }
    h->stream_bytes = 0;
}

}  // namespace cdtw

using namespace cdtw;

extern "C" {

int cdtw_stream_begin(cdtw_handle h, const float* h_query, int M, int W, int metric,
                      int64_t chunk) {
    if (!h) return CDTW_EINVAL;
    if (!h_query) return set_error(h, CDTW_EINVAL, "null query");
    if (metric != CDTW_EUCLIDEAN && metric != CDTW_MANHATTAN)
        return set_error(h, CDTW_EINVAL, "bad metric %d", metric);
    if (M < 11 || M > CDTW_MAX_QUERY)
        return set_error(h, CDTW_EINVAL, "query length %d outside [11, %d]", M, CDTW_MAX_QUERY);
    if (W < 0) return set_error(h, CDTW_EINVAL, "negative band %d", W);
    const int64_t C = chunk > 0 ? chunk : kStreamChunkDefault;
    if (C < M || C + M > INT32_MAX)
        return set_error(h, CDTW_EINVAL, "chunk of %lld samples for M=%d", (long long)C, M);
    CDTW_CUDA(h, cudaSetDevice(h->device));
    StreamState* s = state(h);
    if (s && s->active) {
        // a stream that was begun and never ended: its work is dropped
        CDTW_CUDA(h, cudaStreamSynchronize(h->stream));
        CDTW_CUDA(h, cudaStreamSynchronize(s->copy));
    }
    if (s) s->finish();
    CDTW_TRY(cdtw_set_query(h, h_query, M, W, CDTW_HOST));
    if (!s) {
        s = new (std::nothrow) StreamState();
        if (!s) return set_error(h, CDTW_ENOMEM, "stream state");
        h->stream_state = s;
    }
    s->M = M;
    s->W = std::min(W, M - 1);
    s->metric = metric;
    s->C = C;
    const int64_t N = C + M - 1, Nw = C;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off = (size_t)round_up((int64_t)(off + bytes), 256);
        return o;
    };
    const size_t o_d0 = take(sizeof(float) * N), o_d1 = take(sizeof(float) * N);
    const size_t o_mu = take(sizeof(double) * Nw), o_sg = take(sizeof(float) * Nw);
    const size_t o_best = take(sizeof(StreamBest));
    const size_t o_ws = take(search_workspace_bytes(N, M, s->W));
    // buffers of an earlier stream are reused when large enough (its work
    // has finished: the end of a stream synchronises)
    int st = CDTW_OK;
    if (s->dbytes < off) {
        st = check_memory_limit(h, s->dbytes, off, "stream buffers");
        if (st == CDTW_OK && s->dmem) {
            st = check_cuda(h, cudaFree(s->dmem), "cudaFree(stream)");
            s->dmem = nullptr;
            s->dbytes = 0;
            h->stream_bytes = 0;
        }
        if (st == CDTW_OK) st = check_cuda(h, cudaMalloc(&s->dmem, off), "cudaMalloc(stream)");
        if (st == CDTW_OK) {
            s->dbytes = off;
            h->stream_bytes = off;
        }
    }
    if (st == CDTW_OK && s->scap < C) {
        s->free_stage();
        for (int b = 0; st == CDTW_OK && b < 2; ++b)
            st = check_cuda(h, cudaMallocHost(&s->stage[b], sizeof(float) * C), "cudaMallocHost");
        if (st == CDTW_OK) s->scap = C;
    }
    for (int b = 0; st == CDTW_OK && b < 2; ++b) {
        if (!s->staged[b])
            st = check_cuda(h, cudaEventCreateWithFlags(&s->staged[b], cudaEventDisableTiming),
                            "event");
        if (st == CDTW_OK && !s->done[b])
            st = check_cuda(h, cudaEventCreateWithFlags(&s->done[b], cudaEventDisableTiming),
                            "event");
        if (st == CDTW_OK && !s->copied[b])
            st = check_cuda(h, cudaEventCreateWithFlags(&s->copied[b], cudaEventDisableTiming),
                            "event");
    }
    if (st == CDTW_OK && !s->pushed)
        st = check_cuda(h, cudaEventCreateWithFlags(&s->pushed, cudaEventDisableTiming), "event");
    if (st == CDTW_OK && !s->copy)
        st = check_cuda(h, cudaStreamCreateWithFlags(&s->copy, cudaStreamNonBlocking), "stream");
    if (st != CDTW_OK) {
        stream_release(h);
        return st;
    }
    s->active = true;
    char* base = (char*)s->dmem;
    s->dbuf[0] = (float*)(base + o_d0);
    s->dbuf[1] = (float*)(base + o_d1);
    s->mu = (double*)(base + o_mu);
    s->sigma = (float*)(base + o_sg);
    s->best = (StreamBest*)(base + o_best);
    s->sws = base + o_ws;
    // the copy stream starts after the query preparation on the handle's stream
    cudaEvent_t ev = s->done[0];
    CDTW_CUDA(h, cudaEventRecord(ev, h->stream));
    CDTW_CUDA(h, cudaStreamWaitEvent(s->copy, ev, 0));
    stream_init_kernel<<<1, 1, 0, h->stream>>>(s->best);
    CDTW_LAUNCH(h, "stream_init_kernel");
    return CDTW_OK;
}

int cdtw_stream_push(cdtw_handle h, const float* h_samples, int64_t n) {
    if (!h) return CDTW_EINVAL;
    StreamState* s = state(h);
    if (!s || !s->active) return set_error(h, CDTW_EINVAL, "no stream begun (cdtw_stream_begin)");
    if (n < 0 || (n > 0 && !h_samples)) return set_error(h, CDTW_EINVAL, "bad samples");
    if (n == 0) return CDTW_OK;
    CDTW_CUDA(h, cudaSetDevice(h->device));
    // samples go straight into the current device chunk: from page-locked
    // memory by one copy (waited for before returning, the caller may reuse
    // its buffer), else through the two pinned staging buffers in turn
    const bool pinned = page_locked(h_samples);
    while (n > 0) {
        // a device buffer is refilled after its previous chunk's search
        if (s->fill == 0 && s->used[s->cur])
            CDTW_CUDA(h, cudaStreamWaitEvent(s->copy, s->done[s->cur], 0));
        const int64_t take = std::min(n, s->C - s->fill);
        float* dst = s->dbuf[s->cur] + (s->M - 1) + s->fill;
        if (pinned) {
            CDTW_CUDA(h, cudaMemcpyAsync(dst, h_samples, sizeof(float) * take,
                                         cudaMemcpyHostToDevice, s->copy));
        } else {
            for (int64_t a = 0; a < take;) {
                const int64_t part = std::min(take - a, s->scap);
                const int sl = s->slot;
                // a staging buffer is free once its last copy has left it
                if (s->slot_used[sl]) CDTW_CUDA(h, cudaEventSynchronize(s->staged[sl]));
                memcpy(s->stage[sl], h_samples + a, sizeof(float) * part);
                CDTW_CUDA(h, cudaMemcpyAsync(dst + a, s->stage[sl], sizeof(float) * part,
                                             cudaMemcpyHostToDevice, s->copy));
                CDTW_CUDA(h, cudaEventRecord(s->staged[sl], s->copy));
                s->slot_used[sl] = true;
                s->slot ^= 1;
                a += part;
            }
        }
        s->fill += take;
        s->total += take;
        h_samples += take;
        n -= take;
        if (s->fill == s->C) {
            CDTW_TRY(launch_chunk(h, *s, s->C));
            s->fill = 0;
            s->cur ^= 1;
        }
    }
    if (pinned) {
        CDTW_CUDA(h, cudaEventRecord(s->pushed, s->copy));
        CDTW_CUDA(h, cudaEventSynchronize(s->pushed));
    }
    return CDTW_OK;
}

int cdtw_stream_end(cdtw_handle h, int64_t* location, float* distance, int64_t* scanned) {
    if (!h) return CDTW_EINVAL;
    StreamState* s = state(h);
    if (!s || !s->active) return set_error(h, CDTW_EINVAL, "no stream begun (cdtw_stream_begin)");
    CDTW_CUDA(h, cudaSetDevice(h->device));
    int st = CDTW_OK;
    if (s->fill > 0) {
        if (s->chunks > 0 || s->fill >= s->M) st = launch_chunk(h, *s, s->fill);
        s->fill = 0;
    }
    StreamBest b;
    if (st == CDTW_OK)
        st = check_cuda(h, cudaMemcpyAsync(h->pinned, s->best, sizeof(StreamBest),
                                           cudaMemcpyDeviceToHost, h->stream),
                        "cudaMemcpyAsync");
    if (st == CDTW_OK) st = check_cuda(h, cudaStreamSynchronize(h->stream), "sync");
    if (st == CDTW_OK) memcpy(&b, h->pinned, sizeof(b));
    const int64_t total = s->total;
    const int M = s->M, metric = s->metric;
    if (st != CDTW_OK) {
        stream_release(h);
        return st;
    }
    s->finish();
    if (scanned) *scanned = total;
    if (total < M) return set_error(h, CDTW_EINVAL, "stream of %lld samples is shorter than the query",
                                    (long long)total);
    if (b.loc < 0)
        return set_error(h, CDTW_EINVAL,
                         "no window has a finite distance (NaN or Inf in the query or the stream)");
    const uint32_t bits = (uint32_t)(b.carried >> 32);
    float d;
    memcpy(&d, &bits, 4);
    h->last_counts[0] = total - M + 1;
    h->last_counts[1] = b.n1;
    h->last_counts[2] = b.n2;
    h->last_flag = bits < b.kmax ? 1 : 0;
    if (location) *location = (int64_t)b.loc;
    if (distance) *distance = metric == CDTW_EUCLIDEAN ? sqrtf(d) : d;
    return CDTW_OK;
}

}  // extern "C"
