// Batched search as concurrent single-query pipelines in one CUDA graph
// (cdtw_search_batched without tile shapes).
//
// Each query runs the same device pipeline as cdtw_prune_cdtw -- query
// preparation, window statistics, LB_Kim, LB_Keogh, the early-abandoning or
// wavefront cDTW -- so its result is bit-identical to the single-query
// search, and every improvement of that path serves the batch too.  The
// queries are spread over K internal work contexts ("lanes": a stream, a
// query pack, statistics and a search work area each) by longest-first
// greedy assignment on the band cells M(2W+1); a lane runs its queries in
// (length, band) order, so queries of one length share their window
// statistics.  The whole batch -- the copy of the query values, every lane's
// queries, the copy of the result keys back -- is captured once in a CUDA
// graph (fork and join through events) and replayed while the subject, the
// lengths, bands and metric stay the same; the host synchronises once per
// call.  The first call of a shape runs the lanes eagerly (sizing any
// buffer a kernel family grows on first use) before the capture.
#include "common.cuh"

#include <algorithm>
#include <new>
#include <numeric>

namespace cdtw {

namespace {

constexpr int kPipeLanes = 16;

struct PipePlan {
    const float* subject = nullptr;
    int64_t N = 0;
    int metric = -1;
    std::vector<int> Ms, Ws;
    int nq = 0, K = 0;
    std::vector<cdtw_handle_s*> lanes;
    std::vector<std::vector<int>> lane_queries;  // per lane, in (M, W) order
    std::vector<char*> lane_mem;                 // pack | mu | sigma | search work area
    std::vector<size_t> lane_pack_bytes, lane_stats_off, lane_sigma_off, lane_ws_off;
    void* dmem = nullptr;
    float* draw = nullptr;                  // query values, concatenated
    std::vector<int64_t> raw_off;
    size_t raw_floats = 0;
    unsigned long long* dkeys = nullptr;    // result key per query
    void* hpin = nullptr;                   // staging: query values, then the keys
    cudaStream_t master = nullptr;
    cudaEvent_t fork = nullptr, in = nullptr;
    std::vector<cudaEvent_t> joins;
    cudaGraphExec_t exec = nullptr;

    void release() {
        if (master) cudaStreamSynchronize(master);
        for (cdtw_handle_s* l : lanes) {
            if (l->stream) cudaStreamSynchronize(l->stream);
            if (l->ring) cudaFree(l->ring);
            if (l->own_stream) cudaStreamDestroy(l->own_stream);
            delete l;
        }
        if (exec) cudaGraphExecDestroy(exec);
        if (dmem) cudaFree(dmem);
        if (hpin) cudaFreeHost(hpin);
        if (fork) cudaEventDestroy(fork);
        if (in) cudaEventDestroy(in);
        for (cudaEvent_t e : joins) cudaEventDestroy(e);
        if (master) cudaStreamDestroy(master);
        *this = PipePlan();
    }
};

size_t round256(size_t b) { return (b + 255) / 256 * 256; }

// A lane's queries: prepare, statistics (once per length in a row), search,
// result key to dkeys[q].
int run_lane(cdtw_handle_s* l, PipePlan& p, int li, bool euclid) {
    char* base = p.lane_mem[li];
    double* mu = (double*)(base + p.lane_stats_off[li]);
    float* sigma = (float*)(base + p.lane_sigma_off[li]);
    char* ws = base + p.lane_ws_off[li];
    int last_m = -1;
    for (int q : p.lane_queries[li]) {
        const int M = p.Ms[q], W = p.Ws[q];
        query_pack_layout(M, W, &l->q, base);
        l->has_query = true;
        CDTW_TRY(launch_prepare_query(l, p.draw + p.raw_off[q], M, W));
        if (M != last_m) {
            CDTW_TRY(launch_avg_std(l, p.subject, p.N, M, mu, sigma));
            last_m = M;
        }
        unsigned long long* key;
        int* ctr;
        CDTW_TRY(run_search(l, p.subject, p.N, mu, sigma, euclid, ws, &key, &ctr));
        CDTW_CUDA(l, cudaMemcpyAsync(p.dkeys + q, key, sizeof(unsigned long long),
                                     cudaMemcpyDeviceToDevice, l->stream));
    }
    return CDTW_OK;
}

// Enqueues the whole batch on the master stream: query values in, every lane
// forked off and joined back, keys out.
int enqueue(cdtw_handle h, PipePlan& p, bool euclid) {
    CDTW_CUDA(h, cudaMemcpyAsync(p.draw, p.hpin, p.raw_floats * sizeof(float),
                                 cudaMemcpyHostToDevice, p.master));
    CDTW_CUDA(h, cudaEventRecord(p.fork, p.master));
    for (int li = 0; li < p.K; ++li) {
        cdtw_handle_s* l = p.lanes[li];
        CDTW_CUDA(h, cudaStreamWaitEvent(l->stream, p.fork, 0));
        const int st = run_lane(l, p, li, euclid);
        if (st != CDTW_OK) return set_error(h, st, "batched lane %d: %s", li, l->err);
        CDTW_CUDA(h, cudaEventRecord(p.joins[li], l->stream));
        CDTW_CUDA(h, cudaStreamWaitEvent(p.master, p.joins[li], 0));
    }
    char* keys_h = (char*)p.hpin + round256(p.raw_floats * sizeof(float));
    CDTW_CUDA(h, cudaMemcpyAsync(keys_h, p.dkeys, sizeof(unsigned long long) * p.nq,
                                 cudaMemcpyDeviceToHost, p.master));
    return CDTW_OK;
}

int build(cdtw_handle h, PipePlan& p, bool euclid) {
    const int nq = p.nq;
    p.K = std::min(kPipeLanes, nq);
    // longest-first greedy assignment on the band cells
    std::vector<int> ord(nq);
    std::iota(ord.begin(), ord.end(), 0);
    auto cost = [&](int q) { return (double)p.Ms[q] * (2.0 * p.Ws[q] + 1.0); };
    std::sort(ord.begin(), ord.end(), [&](int a, int b) { return cost(a) > cost(b); });
    std::vector<double> load(p.K, 0.0);
    p.lane_queries.assign(p.K, {});
    for (int q : ord) {
        const int li = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        load[li] += cost(q);
        p.lane_queries[li].push_back(q);
    }
    for (auto& v : p.lane_queries)
        std::sort(v.begin(), v.end(), [&](int a, int b) {
            return p.Ms[a] != p.Ms[b] ? p.Ms[a] < p.Ms[b] : (p.Ws[a] != p.Ws[b] ? p.Ws[a] < p.Ws[b] : a < b);
        });
    // device memory: query values, keys, and per lane pack | stats | work area
    p.raw_off.resize(nq);
    p.raw_floats = 0;
    for (int q = 0; q < nq; ++q) {
        p.raw_off[q] = (int64_t)p.raw_floats;
        p.raw_floats += (size_t)p.Ms[q];
    }
    size_t off = 0;
    const size_t o_raw = off;
    off += round256(p.raw_floats * sizeof(float));
    const size_t o_keys = off;
    off += round256(sizeof(unsigned long long) * nq);
    std::vector<size_t> o_lane(p.K);
    p.lane_pack_bytes.assign(p.K, 0);
    p.lane_stats_off.assign(p.K, 0);
    p.lane_sigma_off.assign(p.K, 0);
    p.lane_ws_off.assign(p.K, 0);
    for (int li = 0; li < p.K; ++li) {
        size_t pack = 0, wsb = 0;
        int mmin = 1 << 30;
        for (int q : p.lane_queries[li]) {
            pack = std::max(pack, query_pack_layout(p.Ms[q], p.Ws[q], nullptr, nullptr));
            wsb = std::max(wsb, search_workspace_bytes(p.N, p.Ms[q], p.Ws[q]));
            mmin = std::min(mmin, p.Ms[q]);
        }
        const int64_t nw = p.N - mmin + 1;
        o_lane[li] = off;
        p.lane_stats_off[li] = round256(pack);
        p.lane_sigma_off[li] = p.lane_stats_off[li] + round256(sizeof(double) * nw);
        p.lane_ws_off[li] = p.lane_sigma_off[li] + round256(sizeof(float) * nw);
        off += p.lane_ws_off[li] + round256(wsb);
    }
    CDTW_TRY(check_memory_limit(h, h->batch_bytes, off, "batched-search lanes"));
    CDTW_CUDA(h, cudaMalloc(&p.dmem, off));
    h->batch_bytes = off;
    char* d = (char*)p.dmem;
    p.draw = (float*)(d + o_raw);
    p.dkeys = (unsigned long long*)(d + o_keys);
    p.lane_mem.resize(p.K);
    for (int li = 0; li < p.K; ++li) p.lane_mem[li] = d + o_lane[li];
    CDTW_CUDA(h, cudaMallocHost(&p.hpin, round256(p.raw_floats * sizeof(float)) +
                                             sizeof(unsigned long long) * nq));
    CDTW_CUDA(h, cudaStreamCreateWithFlags(&p.master, cudaStreamNonBlocking));
    CDTW_CUDA(h, cudaEventCreateWithFlags(&p.fork, cudaEventDisableTiming));
    CDTW_CUDA(h, cudaEventCreateWithFlags(&p.in, cudaEventDisableTiming));
    p.joins.assign(p.K, nullptr);
    for (auto& e : p.joins) CDTW_CUDA(h, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (int li = 0; li < p.K; ++li) {
        cdtw_handle_s* l = new (std::nothrow) cdtw_handle_s();
        if (!l) return set_error(h, CDTW_ENOMEM, "batched lane");
        p.lanes.push_back(l);
        l->device = h->device;
        l->sm_count = h->sm_count;
        memcpy(l->band_variant, h->band_variant, sizeof(l->band_variant));
        CDTW_CUDA(h, cudaStreamCreateWithFlags(&l->own_stream, cudaStreamNonBlocking));
        l->stream = l->own_stream;
    }
    return CDTW_OK;
}

}  // namespace

void batch_pipe_release(cdtw_handle h) {
    PipePlan* p = reinterpret_cast<PipePlan*>(h->batch_pipe);
    if (p) {
        p->release();
        delete p;
        h->batch_pipe = nullptr;
        h->batch_bytes = 0;
    }
}

// Batched search through concurrent single-query pipelines (see above).
int search_batched_pipelines(cdtw_handle h, const float* d_subject, int64_t N,
                             const float* h_queries, const std::vector<int>& M,
                             const std::vector<int>& W, int metric, int64_t* locations,
                             float* distances) {
    const int nq = (int)M.size();
    const bool euclid = metric == CDTW_EUCLIDEAN;
    batch_plan_release(h);  // the tile-mode plan and this one share the memory budget
    PipePlan*& pp = *reinterpret_cast<PipePlan**>(&h->batch_pipe);
    if (!pp) pp = new (std::nothrow) PipePlan();
    if (!pp) return set_error(h, CDTW_ENOMEM, "batched plan");
    PipePlan& p = *pp;
    const bool same = p.exec && p.subject == d_subject && p.N == N && p.metric == metric &&
                      p.Ms == M && p.Ws == W;
    bool fresh = false;
    if (!same) {
        p.release();
        h->batch_bytes = 0;
        p.subject = d_subject;
        p.N = N;
        p.metric = metric;
        p.Ms = M;
        p.Ws = W;
        p.nq = nq;
        int st = build(h, p, euclid);
        if (st != CDTW_OK) {
            p.release();
            h->batch_bytes = 0;
            return st;
        }
        fresh = true;
    }
    memcpy(p.hpin, h_queries, p.raw_floats * sizeof(float));
    // ordered after the caller's earlier work on the handle's stream
    CDTW_CUDA(h, cudaEventRecord(p.in, h->stream));
    CDTW_CUDA(h, cudaStreamWaitEvent(p.master, p.in, 0));
    if (fresh) {
        // eager first run (grows any work buffer a kernel family sizes on its
        // first launch), then the capture replayed from the next call on
        int st = enqueue(h, p, euclid);
        if (st == CDTW_OK) st = check_cuda(h, cudaStreamSynchronize(p.master), "batched run");
        if (st != CDTW_OK) {
            p.release();
            h->batch_bytes = 0;
            return st;
        }
        cudaGraph_t g = nullptr;
        CDTW_CUDA(h, cudaStreamBeginCapture(p.master, cudaStreamCaptureModeRelaxed));
        st = enqueue(h, p, euclid);
        const cudaError_t ce = cudaStreamEndCapture(p.master, &g);
        if (st != CDTW_OK || ce != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            p.release();
            h->batch_bytes = 0;
            return st != CDTW_OK ? st : check_cuda(h, ce, "cudaStreamEndCapture");
        }
        const cudaError_t ie = cudaGraphInstantiate(&p.exec, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) {
            p.release();
            h->batch_bytes = 0;
            return check_cuda(h, ie, "cudaGraphInstantiate");
        }
    } else {
        CDTW_CUDA(h, cudaGraphLaunch(p.exec, p.master));
        CDTW_CUDA(h, cudaStreamSynchronize(p.master));
    }
    CDTW_CUDA(h, cudaEventRecord(p.in, p.master));
    CDTW_CUDA(h, cudaStreamWaitEvent(h->stream, p.in, 0));
    const unsigned long long* keys =
        (const unsigned long long*)((char*)p.hpin + round256(p.raw_floats * sizeof(float)));
    for (int q = 0; q < nq; ++q) {
        const unsigned long long k = keys[q];
        if (k == ~0ull || (uint32_t)k == 0xffffffffu) {
            locations[q] = -1;
            distances[q] = INFINITY;
            continue;
        }
        const uint32_t bits = (uint32_t)(k >> 32);
        float dd;
        memcpy(&dd, &bits, 4);
        locations[q] = (int64_t)(uint32_t)k;
        distances[q] = euclid ? sqrtf(dd) : dd;
    }
    return CDTW_OK;
}

}  // namespace cdtw
