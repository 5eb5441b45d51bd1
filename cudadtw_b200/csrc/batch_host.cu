// Host side of the batched search: work lists, query packs, rings, and the
// CUDA graph that replays the whole batch (query upload, query preparation,
// the three persistent passes of batch.cu, result read-back) in one launch.
// The graph is cached on the handle and replayed while the subject, the
// query lengths/bands and the tile shapes stay the same; only the query
// values change between calls.
#include "batch.cuh"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace cdtw {

struct BatchPlan {
    // identity of the cached plan
    const float* subject = nullptr;
    int64_t N = 0;
    int metric = -1;
    std::vector<int> Ms, Ws, Rs, Ts;
    int lane_refill = 0;
    // device memory (one allocation) and pinned staging
    void* dmem = nullptr;
    void* hpin = nullptr;
    size_t raw_floats = 0;
    unsigned long long* dkeys = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    int nq = 0;
    void release() {
        if (exec) cudaGraphExecDestroy(exec);
        if (dmem) cudaFree(dmem);
        if (hpin) cudaFreeHost(hpin);
        if (ev_in) cudaEventDestroy(ev_in);
        if (ev_out) cudaEventDestroy(ev_out);
        *this = BatchPlan();
    }
};

static int default_rows(int W) {
    int r = 1;
    while (r * 2 <= std::min(16, W + 1)) r *= 2;
    return r;
}

// rows[q] == 0: register-band main pass (W <= 96); else strip rows.
static int build_plan(cdtw_handle h, BatchPlan& p, bool euclid) {
    const int nq = (int)p.Ms.size();
    const int64_t N = p.N;
    int mmax = 0, tmax = 0, pmax = 0, lq4max = 0;
    std::vector<int> ntiles(nq), seed_rows(nq), groups(nq);
    for (int q = 0; q < nq; ++q) {
        const int M = p.Ms[q], W = p.Ws[q], T = p.Ts[q];
        ntiles[q] = (int)div_up(N - M + 1, T);
        seed_rows[q] = p.Rs[q] ? p.Rs[q] : default_rows(W);
        groups[q] = (int)std::max<int64_t>(1, div_up(ntiles[q], seed_target(M, W)));
        mmax = std::max(mmax, M);
        tmax = std::max(tmax, T);
        pmax = std::max(pmax, (int)round_up(2 * W + 2, seed_rows[q]));
        if (p.Rs[q] == 0) lq4max = std::max(lq4max, (int)round_up(M + 2 * W + 8, 4) / 4);
    }
    // launches: seed pass + seed cDTW over all queries; main pass per bucket
    std::vector<int> all(nq);
    for (int q = 0; q < nq; ++q) all[q] = q;
    std::vector<std::vector<int>> buckets;  // [0] strip, then one per register band
    std::vector<int> bucket_w;              // -1 for strip
    buckets.push_back({});
    bucket_w.push_back(-1);
    for (int q = 0; q < nq; ++q) {
        if (p.Rs[q] != 0) {
            buckets[0].push_back(q);
            continue;
        }
        size_t k = 1;
        while (k < bucket_w.size() && bucket_w[k] != p.Ws[q]) ++k;
        if (k == bucket_w.size()) {
            buckets.push_back({});
            bucket_w.push_back(p.Ws[q]);
        }
        buckets[k].push_back(q);
    }
    const size_t smem = batch_smem_bytes(tmax, mmax, lq4max);
    if (smem > 227 * 1024)
        return set_error(h, CDTW_EUNSUPPORTED, "batch tile too large for shared memory");
    int blocks = 0;
    CDTW_TRY(batch_grid(h, euclid, smem, &blocks));
    std::vector<int> reg_blocks(buckets.size(), 0);
    for (size_t k = 1; k < buckets.size(); ++k)
        CDTW_TRY(batch_reg_prepare(h, bucket_w[k], euclid, smem, &reg_blocks[k]));
    const int ring_stride = pmax * 32;
    // one device allocation, carved
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off = (size_t)round_up((int64_t)(off + bytes), 256);
        return o;
    };
    size_t raw_floats = 0;
    std::vector<int64_t> raw_off(nq);
    for (int q = 0; q < nq; ++q) {
        raw_off[q] = (int64_t)raw_floats;
        raw_floats += (size_t)p.Ms[q];
    }
    const size_t o_raw = take(raw_floats * sizeof(float));
    const size_t o_rawoff = take(nq * sizeof(int64_t));
    std::vector<size_t> pack_off(nq);
    std::vector<int> lqr(nq), lq(nq);
    for (int q = 0; q < nq; ++q) {
        const int M = p.Ms[q], W = p.Ws[q];
        lqr[q] = qrev_len(M, W);
        lq[q] = p.Rs[q] == 0 ? (int)round_up(M + 2 * W + 8, 4) : 0;
        pack_off[q] = take(sizeof(float2) * M + sizeof(float) * M + sizeof(double) * M +
                           sizeof(float) * 4 * ((size_t)lqr[q] + lq[q]) + 1024);
    }
    const size_t o_packs = take(sizeof(QueryPack) * nq);
    const size_t o_qs = take(sizeof(BatchQ) * nq);
    // per launch: qsel, item prefix, chunk prefix
    const int nl = (int)buckets.size() + 1;  // launch 0: seed (all), 1..: main buckets
    std::vector<std::vector<int>> lsel(nl), lip(nl), lcp(nl);
    lsel[0] = all;
    for (size_t k = 0; k < buckets.size(); ++k) lsel[k + 1] = buckets[k];
    for (int l = 0; l < nl; ++l) {
        lip[l].assign(lsel[l].size() + 1, 0);
        lcp[l].assign(lsel[l].size() + 1, 0);
        for (size_t i = 0; i < lsel[l].size(); ++i) {
            const int q = lsel[l][i];
            lip[l][i + 1] = lip[l][i] + ntiles[q];
            lcp[l][i + 1] = lcp[l][i] + (int)div_up(div_up(ntiles[q], groups[q]), 32);
        }
    }
    std::vector<size_t> o_sel(nl), o_ip(nl), o_cp(nl);
    for (int l = 0; l < nl; ++l) {
        o_sel[l] = take(sizeof(int) * std::max<size_t>(1, lsel[l].size()));
        o_ip[l] = take(sizeof(int) * (lsel[l].size() + 1));
        o_cp[l] = take(sizeof(int) * (lsel[l].size() + 1));
    }
    const int n_seed_items = lip[0][nq];
    const size_t o_seeds = take(sizeof(SeedRec) * (size_t)n_seed_items);
    const size_t o_keys = take(sizeof(unsigned long long) * nq);
    const size_t o_ctr = take(sizeof(int) * (2 + nl));
    const size_t o_ring =
        take((size_t)blocks * batch_warps_per_block() * ring_stride * sizeof(float));
    CDTW_TRY(check_memory_limit(h, h->batch_bytes, off, "batched-search plan"));
    CDTW_CUDA(h, cudaMalloc(&p.dmem, off));
    h->batch_bytes = off;
    CDTW_CUDA(h, cudaMallocHost(&p.hpin, raw_floats * sizeof(float) + nq * 8 + 64));
    p.raw_floats = raw_floats;
    char* d = (char*)p.dmem;
    // host images of the descriptors
    std::vector<QueryPack> packs(nq);
    std::vector<BatchQ> qs(nq);
    for (int q = 0; q < nq; ++q) {
        const int M = p.Ms[q], W = p.Ws[q];
        char* bp = d + pack_off[q];
        QueryPack& k = packs[q];
        k.M = M;
        k.W = W;
        k.env = (float2*)bp;
        k.zq = (float*)(bp + sizeof(float2) * M);
        k.zq64 = (double*)(((uintptr_t)(bp + sizeof(float2) * M + sizeof(float) * M) + 7) &
                           ~(uintptr_t)7);
        k.lqr = lqr[q];
        k.qrev_base = qrev_hi(M, W);
        k.qrev = (float*)(((uintptr_t)(k.zq64 + M) + 15) & ~(uintptr_t)15);
        k.lq = lq[q];
        k.qpad = lq[q] ? k.qrev + 4 * (size_t)lqr[q] : nullptr;
        BatchQ& Q = qs[q];
        memset(&Q, 0, sizeof(Q));
        Q.sa.x = p.subject;
        Q.sa.qrev4 = (const float4*)k.qrev;
        Q.sa.qrev0 = k.qrev;
        Q.sa.lqr4 = k.lqr / 4;
        Q.sa.qbase = k.qrev_base;
        Q.sa.M = M;
        Q.sa.W = W;
        Q.sa.P = (int)round_up(2 * W + 2, seed_rows[q]);
        Q.sa.Nw = (int)(N - M + 1);
        Q.zq = k.zq;
        Q.env = k.env;
        Q.qpad4 = (const float4*)k.qpad;
        Q.lq4 = lq[q] / 4;
        Q.key = (unsigned long long*)(d + o_keys) + q;
        Q.R = seed_rows[q];
        Q.T = p.Ts[q];
        Q.Nw = (int)(N - M + 1);
        Q.ntiles = ntiles[q];
        Q.item0 = lip[0][q];
        Q.chunk0 = lcp[0][q];
        Q.seed_group = groups[q];
        Q.lane_refill = p.lane_refill;
    }
    CDTW_CUDA(h, cudaMemcpy(d + o_rawoff, raw_off.data(), nq * sizeof(int64_t),
                            cudaMemcpyHostToDevice));
    CDTW_CUDA(h, cudaMemcpy(d + o_packs, packs.data(), sizeof(QueryPack) * nq,
                            cudaMemcpyHostToDevice));
    CDTW_CUDA(h, cudaMemcpy(d + o_qs, qs.data(), sizeof(BatchQ) * nq, cudaMemcpyHostToDevice));
    for (int l = 0; l < nl; ++l) {
        if (!lsel[l].empty())
            CDTW_CUDA(h, cudaMemcpy(d + o_sel[l], lsel[l].data(), sizeof(int) * lsel[l].size(),
                                    cudaMemcpyHostToDevice));
        CDTW_CUDA(h, cudaMemcpy(d + o_ip[l], lip[l].data(), sizeof(int) * lip[l].size(),
                                cudaMemcpyHostToDevice));
        CDTW_CUDA(h, cudaMemcpy(d + o_cp[l], lcp[l].data(), sizeof(int) * lcp[l].size(),
                                cudaMemcpyHostToDevice));
    }
    auto args = [&](int l, int ctr_idx) {
        BatchArgs a;
        a.qs = (const BatchQ*)(d + o_qs);
        a.qsel = (const int*)(d + o_sel[l]);
        a.nq = (int)lsel[l].size();
        a.item_prefix = (const int*)(d + o_ip[l]);
        a.chunk_prefix = (const int*)(d + o_cp[l]);
        a.n_items = lip[l].back();
        a.n_chunks = lcp[l].back();
        a.ctr = (int*)(d + o_ctr);
        a.ctr_idx = ctr_idx;
        a.seeds = (SeedRec*)(d + o_seeds);
        a.ring = (float*)(d + o_ring);
        a.ring_stride = ring_stride;
        a.x = p.subject;
        a.tmax = tmax;
        a.mmax = mmax;
        a.lq4max = lq4max;
        return a;
    };
    p.dkeys = (unsigned long long*)(d + o_keys);
    // capture on the handle's own (capturable) stream
    cudaStream_t user = h->stream;
    cudaStream_t cs = h->own_stream;
    h->stream = cs;
    cudaGraph_t g = nullptr;
    int st = CDTW_OK;
    if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        h->stream = user;
        return check_cuda(h, cudaGetLastError(), "cudaStreamBeginCapture");
    }
    cudaMemcpyAsync(d + o_raw, p.hpin, raw_floats * sizeof(float), cudaMemcpyHostToDevice, cs);
    st = launch_prepare_queries(h, (const float*)(d + o_raw), (const int64_t*)(d + o_rawoff),
                                (const QueryPack*)(d + o_packs), nq, mmax);
    cudaMemsetAsync(d + o_keys, 0xff, sizeof(unsigned long long) * nq, cs);
    cudaMemsetAsync(d + o_ctr, 0, sizeof(int) * (2 + nl), cs);
    if (st == CDTW_OK) st = launch_batch_seed(h, args(0, 0), args(0, 1), euclid, smem, blocks);
    for (size_t k = 0; st == CDTW_OK && k < buckets.size(); ++k) {
        if (buckets[k].empty()) continue;
        const BatchArgs a = args((int)k + 1, 2 + (int)k);
        st = (bucket_w[k] < 0) ? launch_batch_strip(h, a, euclid, smem, blocks)
                               : launch_batch_reg(h, a, bucket_w[k], euclid, smem, reg_blocks[k]);
    }
    cudaMemcpyAsync((char*)p.hpin + raw_floats * sizeof(float), d + o_keys,
                    sizeof(unsigned long long) * nq, cudaMemcpyDeviceToHost, cs);
    const cudaError_t ce = cudaStreamEndCapture(cs, &g);
    h->stream = user;
    if (st != CDTW_OK) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (ce != cudaSuccess) return check_cuda(h, ce, "cudaStreamEndCapture");
    const cudaError_t ie = cudaGraphInstantiate(&p.exec, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) return check_cuda(h, ie, "cudaGraphInstantiate");
    CDTW_CUDA(h, cudaEventCreateWithFlags(&p.ev_in, cudaEventDisableTiming));
    CDTW_CUDA(h, cudaEventCreateWithFlags(&p.ev_out, cudaEventDisableTiming));
    p.nq = nq;
    return CDTW_OK;
}

}  // namespace cdtw

using namespace cdtw;

extern "C" int cdtw_search_batched(cdtw_handle h, const float* d_subject, int64_t N,
                                   const float* h_queries, const int* Ms, const int* Ws, int nq,
                                   int metric, const int* rows, const int* tiles,
                                   int64_t* locations, float* distances) {
    if (!h) return CDTW_EINVAL;
    if (!d_subject || !h_queries || !Ms || !Ws || !locations || !distances || nq < 1)
        return set_error(h, CDTW_EINVAL, "null pointer or empty batch");
    if (metric != CDTW_EUCLIDEAN && metric != CDTW_MANHATTAN)
        return set_error(h, CDTW_EINVAL, "bad metric %d", metric);
    if (!rows && !tiles) {
        // no tile shapes: concurrent single-query pipelines (batch_pipe.cu)
        std::vector<int> M(Ms, Ms + nq), W(nq);
        for (int q = 0; q < nq; ++q) {
            if (M[q] < 11 || M[q] > CDTW_MAX_QUERY || M[q] > N)
                return set_error(h, CDTW_EINVAL, "query %d: length %d outside [11, min(%d, N)]",
                                 q, M[q], CDTW_MAX_QUERY);
            if (Ws[q] < 0) return set_error(h, CDTW_EINVAL, "query %d: negative band", q);
            W[q] = std::min(Ws[q], M[q] - 1);
        }
        if (N - 1 > INT32_MAX) return set_error(h, CDTW_EUNSUPPORTED, "subject too long");
        CDTW_CUDA(h, cudaSetDevice(h->device));
        return search_batched_pipelines(h, d_subject, N, h_queries, M, W, metric, locations,
                                        distances);
    }
    batch_pipe_release(h);  // the pipelines plan and this one share the memory budget
    std::vector<int> M(Ms, Ms + nq), W(nq), R(nq), T(nq);
    for (int q = 0; q < nq; ++q) {
        if (M[q] < 11 || M[q] > 4096 || M[q] > N)
            return set_error(h, CDTW_EINVAL, "query %d: length %d outside [11, min(4096, N)]", q,
                             M[q]);
        if (Ws[q] < 0) return set_error(h, CDTW_EINVAL, "query %d: negative band", q);
        W[q] = std::min(Ws[q], M[q] - 1);
        // 0 = register-band main pass (W <= 96), else strip rows
        R[q] = rows ? rows[q] : (W[q] <= max_register_band() ? 0 : 16);
        if (R[q] != 0 && R[q] != 1 && R[q] != 2 && R[q] != 4 && R[q] != 8 && R[q] != 16)
            return set_error(h, CDTW_EINVAL, "query %d: rows must be 0, 1, 2, 4, 8 or 16", q);
        if (R[q] == 0 && W[q] > max_register_band()) R[q] = 16;
        if (R[q] > W[q] + 1) R[q] = default_rows(W[q]);
        T[q] = tiles ? tiles[q] : 1024;
        if (T[q] < 32 || T[q] > 4096 || (T[q] & 31))
            return set_error(h, CDTW_EINVAL, "query %d: tile must be a multiple of 32 in [32, 4096]", q);
    }
    if (N - 1 > INT32_MAX) return set_error(h, CDTW_EUNSUPPORTED, "subject too long");
    CDTW_CUDA(h, cudaSetDevice(h->device));
    BatchPlan*& plan = *reinterpret_cast<BatchPlan**>(&h->batch);
    if (!plan) plan = new BatchPlan();
    BatchPlan& p = *plan;
    // strip cDTW refill granularity: per warp unless CDTW_BATCH_LANE_REFILL=1
    const char* lr = getenv("CDTW_BATCH_LANE_REFILL");
    const int lane = (lr && lr[0] == '1') ? 1 : 0;
    const bool same = p.exec && p.subject == d_subject && p.N == N && p.metric == metric &&
                      p.Ms == M && p.Ws == W && p.Rs == R && p.Ts == T && p.lane_refill == lane;
    if (!same) {
        CDTW_CUDA(h, cudaStreamSynchronize(h->own_stream));
        p.release();
        h->batch_bytes = 0;
        p.subject = d_subject;
        p.N = N;
        p.metric = metric;
        p.Ms = M;
        p.Ws = W;
        p.Rs = R;
        p.Ts = T;
        p.lane_refill = lane;
        const int st = build_plan(h, p, metric == CDTW_EUCLIDEAN);
        if (st != CDTW_OK) {
            p.release();
            h->batch_bytes = 0;
            return st;
        }
    }
    // stage the query values, order after the caller's stream, replay
    memcpy(p.hpin, h_queries, p.raw_floats * sizeof(float));
    CDTW_CUDA(h, cudaEventRecord(p.ev_in, h->stream));
    CDTW_CUDA(h, cudaStreamWaitEvent(h->own_stream, p.ev_in, 0));
    CDTW_CUDA(h, cudaGraphLaunch(p.exec, h->own_stream));
    CDTW_CUDA(h, cudaEventRecord(p.ev_out, h->own_stream));
    CDTW_CUDA(h, cudaStreamWaitEvent(h->stream, p.ev_out, 0));
    CDTW_CUDA(h, cudaEventSynchronize(p.ev_out));
    const unsigned long long* keys =
        (const unsigned long long*)((char*)p.hpin + p.raw_floats * sizeof(float));
    for (int q = 0; q < nq; ++q) {
        const unsigned long long k = keys[q];
        if (k == ~0ull) {
            locations[q] = -1;
            distances[q] = INFINITY;
            continue;
        }
        const uint32_t bits = (uint32_t)(k >> 32);
        float dd;
        memcpy(&dd, &bits, 4);
        locations[q] = (int64_t)(uint32_t)k;
        distances[q] = metric == CDTW_EUCLIDEAN ? sqrtf(dd) : dd;
    }
    return CDTW_OK;
}

namespace cdtw {
void batch_plan_release(cdtw_handle h) {
    BatchPlan* p = reinterpret_cast<BatchPlan*>(h->batch);
    if (p) {
        p->release();
        delete p;
        h->batch = nullptr;
        h->batch_bytes = 0;
    }
}
}  // namespace cdtw
