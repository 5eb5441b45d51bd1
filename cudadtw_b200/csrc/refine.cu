// Template refinement (no reference counterpart): Adam steps on query
// templates against their matched stream windows, the whole loop captured as
// one CUDA graph -- against fixed matches (cdtw_refine_templates), or with the
// top-k matches searched again on the device at every step
// (cdtw_refine_templates_search: per template and step the device top-k
// search of run_topk_device, its first k picks gathered as the pair windows).
//
// For template t (length M_t, band W_t) with k matched windows s_j the loss is
// the mean over j of the banded cDTW between the z-normalised template and the
// z-normalised window.  Each step runs, per group of templates of equal
// (M, W): the template broadcast to its k pairs, the pairwise z-normalisation,
// the pairwise forward with path record, the mean loss, the pairwise backward
// (dD = 1/k), and one kernel that sums the k pair gradients of each template
// element and applies Adam (beta1 0.9, beta2 0.999, eps 1e-8).  Groups are
// independent, so their step chains run on up to kBranches forked streams of
// the captured graph.
#include "common.cuh"

#include <algorithm>
#include <cstring>
#include <map>
#include <new>
#include <vector>

namespace cdtw {

namespace {

constexpr int kBranches = 8;
constexpr float kBeta1 = 0.9f, kBeta2 = 0.999f, kEps = 1e-8f;

__global__ void gather_windows_kernel(const float* __restrict__ x, const int64_t* __restrict__ loc,
                                      int64_t n, int L, float* __restrict__ out) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * L) return;
    const int64_t p = e / L;
    out[e] = __ldg(x + loc[p] + (e - p * L));
}

// qrep[(t k + j) L + i] = tmpl[t L + i]
__global__ void broadcast_kernel(const float* __restrict__ tmpl, int nt, int k, int L,
                                 float* __restrict__ qrep) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t total = (int64_t)nt * k * L;
    if (e >= total) return;
    const int64_t p = e / L;
    const int i = (int)(e - p * L);
    qrep[e] = tmpl[(p / k) * L + i];
}

__global__ void fill_kernel(float* __restrict__ a, int64_t n, float v) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n) a[e] = v;
}

// losses[t] = mean of the k pair distances of template t (one warp each)
__global__ void loss_kernel(const float* __restrict__ D, int nt, int k,
                            const int* __restrict__ tid, float* __restrict__ losses) {
    const int t = blockIdx.x;
    if (t >= nt) return;
    double s = 0.0;
    for (int j = threadIdx.x; j < k; j += 32) s += (double)D[(int64_t)t * k + j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) losses[tid[t]] = (float)(s / k);
}

// Sum of the k pair gradients of each template element (they already carry
// dD = 1/k), then one Adam step.  c1 = 1 - beta1^step, c2 = 1 - beta2^step.
__global__ void adam_kernel(const float* __restrict__ dq, int nt, int k, int L,
                            float* __restrict__ tmpl, float* __restrict__ m,
                            float* __restrict__ v, float lr, float c1, float c2) {
    const int t = blockIdx.x;
    const int i = blockIdx.y * blockDim.x + threadIdx.x;
    if (t >= nt || i >= L) return;
    const float* g0 = dq + (int64_t)t * k * L + i;
    double g = 0.0;
    for (int j = 0; j < k; ++j) g += (double)g0[(int64_t)j * L];
    const int64_t e = (int64_t)t * L + i;
    const float gf = (float)g;
    const float mm = kBeta1 * m[e] + (1.f - kBeta1) * gf;
    const float vv = kBeta2 * v[e] + (1.f - kBeta2) * gf * gf;
    m[e] = mm;
    v[e] = vv;
    tmpl[e] -= lr * (mm / c1) / (sqrtf(vv / c2) + kEps);
}

struct Group {
    int L = 0, W = 0;
    std::vector<int> tids;  // template indices
    std::vector<int64_t> toff;  // their offsets in the caller's array
    int nt = 0;
    int64_t n = 0;  // pairs
    float *tmpl, *m, *v, *qrep, *swin, *D, *dq, *dD;
    int64_t* loc;
    int* dtid;
    char* path;
    int branch = 0;
};

inline unsigned blocks_for(int64_t n, int t) { return (unsigned)div_up(n, t); }

// 256-byte aligned slices of one allocation
struct Slices {
    size_t off = 0;
    template <class T>
    size_t take(size_t count) {
        const size_t o = off;
        off = (size_t)round_up((int64_t)(off + count * sizeof(T)), 256);
        return o;
    }
};

}  // namespace

}  // namespace cdtw

using namespace cdtw;

extern "C" int cdtw_refine_templates(cdtw_handle h, const float* d_subject, int64_t N,
                                     float* d_templates, const int* Ms, const int* Ws, int nt,
                                     const int64_t* locations, int k, int steps, float lr,
                                     int metric, float* losses) {
    if (!h) return CDTW_EINVAL;
    if (!d_subject || !d_templates || !Ms || !Ws || !locations || nt < 1 || k < 1 || steps < 0)
        return set_error(h, CDTW_EINVAL, "bad refinement arguments");
    if (metric != CDTW_EUCLIDEAN && metric != CDTW_MANHATTAN)
        return set_error(h, CDTW_EINVAL, "bad metric %d", metric);
    if (!(lr >= 0.f)) return set_error(h, CDTW_EINVAL, "bad learning rate");
    const bool euclid = metric == CDTW_EUCLIDEAN;
    // groups of equal (M, W)
    std::map<std::pair<int, int>, Group> gm;
    int64_t off = 0;
    for (int t = 0; t < nt; ++t) {
        const int M = Ms[t];
        if (M < 2 || M > CDTW_MAX_QUERY || M > N)
            return set_error(h, CDTW_EINVAL, "template %d: length %d", t, M);
        if (Ws[t] < 0) return set_error(h, CDTW_EINVAL, "template %d: negative band", t);
        const int W = std::min(Ws[t], M - 1);
        if (W > CDTW_PAIR_MAX_BAND)
            return set_error(h, CDTW_EUNSUPPORTED, "template %d: band %d exceeds %d", t, W,
                             CDTW_PAIR_MAX_BAND);
        for (int j = 0; j < k; ++j) {
            const int64_t w = locations[(int64_t)t * k + j];
            if (w < 0 || w > N - M)
                return set_error(h, CDTW_EINVAL, "template %d: window %lld outside the subject",
                                 t, (long long)w);
        }
        Group& g = gm[{M, W}];
        g.L = M;
        g.W = W;
        g.tids.push_back(t);
        g.toff.push_back(off);
        off += M;
    }
    std::vector<Group*> groups;
    for (auto& kv : gm) groups.push_back(&kv.second);
    // one allocation: per group its buffers, per branch the pair scratch
    Slices c;
    std::vector<size_t> o_tm, o_m, o_v, o_q, o_s, o_D, o_dq, o_dD, o_loc, o_tid, o_path;
    size_t zmax[kBranches] = {0}, dmax[kBranches] = {0};
    int gi = 0;
    for (Group* g : groups) {
        g->nt = (int)g->tids.size();
        g->n = (int64_t)g->nt * k;
        g->branch = gi++ % kBranches;
        const size_t tl = (size_t)g->nt * g->L, pl = (size_t)g->n * g->L;
        o_tm.push_back(c.take<float>(tl));
        o_m.push_back(c.take<float>(tl));
        o_v.push_back(c.take<float>(tl));
        o_q.push_back(c.take<float>(pl));
        o_s.push_back(c.take<float>(pl));
        o_D.push_back(c.take<float>(g->n));
        o_dq.push_back(c.take<float>(pl));
        o_dD.push_back(c.take<float>(g->n));
        o_loc.push_back(c.take<int64_t>(g->n));
        o_tid.push_back(c.take<int>(g->nt));
        o_path.push_back(c.take<char>(cdtw_pair_path_bytes(g->n, g->L)));
        zmax[g->branch] = std::max(zmax[g->branch], pl);
        dmax[g->branch] = std::max(dmax[g->branch], (size_t)g->n * pair_dirs_words(g->L, g->W));
    }
    const int nb = std::min<int>(kBranches, (int)groups.size());
    size_t o_zq[kBranches], o_zs[kBranches], o_dir[kBranches];
    for (int b = 0; b < nb; ++b) {
        o_zq[b] = c.take<float>(zmax[b]);
        o_zs[b] = c.take<float>(zmax[b]);
        o_dir[b] = c.take<uint32_t>(dmax[b]);
    }
    const size_t o_loss = c.take<float>((size_t)(steps + 1) * nt);
    CDTW_CUDA(h, cudaSetDevice(h->device));
    char* base = nullptr;
    CDTW_TRY(check_memory_limit(h, 0, c.off, "template refinement"));
    CDTW_CUDA(h, cudaMalloc(&base, c.off));
    struct Cleanup {
        char* p;
        std::vector<cudaStream_t> s;
        std::vector<cudaEvent_t> e;
        cudaGraph_t g = nullptr;
        cudaGraphExec_t x = nullptr;
        ~Cleanup() {
            if (x) cudaGraphExecDestroy(x);
            if (g) cudaGraphDestroy(g);
            for (auto ev : e) cudaEventDestroy(ev);
            for (auto st : s) cudaStreamDestroy(st);
            if (p) cudaFree(p);
        }
    } cl{base, {}, {}};
    // set-up (outside the graph): templates in, windows gathered, moments 0
    std::vector<int64_t> hloc;
    std::vector<int> htid;
    for (size_t q = 0; q < groups.size(); ++q) {
        Group& g = *groups[q];
        g.tmpl = (float*)(base + o_tm[q]);
        g.m = (float*)(base + o_m[q]);
        g.v = (float*)(base + o_v[q]);
        g.qrep = (float*)(base + o_q[q]);
        g.swin = (float*)(base + o_s[q]);
        g.D = (float*)(base + o_D[q]);
        g.dq = (float*)(base + o_dq[q]);
        g.dD = (float*)(base + o_dD[q]);
        g.loc = (int64_t*)(base + o_loc[q]);
        g.dtid = (int*)(base + o_tid[q]);
        g.path = base + o_path[q];
        hloc.clear();
        for (int t : g.tids)
            hloc.insert(hloc.end(), locations + (int64_t)t * k, locations + (int64_t)(t + 1) * k);
        CDTW_CUDA(h, cudaMemcpyAsync(g.loc, hloc.data(), sizeof(int64_t) * g.n,
                                     cudaMemcpyHostToDevice, h->stream));
        CDTW_CUDA(h, cudaMemcpyAsync(g.dtid, g.tids.data(), sizeof(int) * g.nt,
                                     cudaMemcpyHostToDevice, h->stream));
        for (int i = 0; i < g.nt; ++i)
            CDTW_CUDA(h, cudaMemcpyAsync(g.tmpl + (size_t)i * g.L, d_templates + g.toff[i],
                                         sizeof(float) * g.L, cudaMemcpyDeviceToDevice,
                                         h->stream));
        CDTW_CUDA(h, cudaMemsetAsync(g.m, 0, sizeof(float) * g.nt * g.L, h->stream));
        CDTW_CUDA(h, cudaMemsetAsync(g.v, 0, sizeof(float) * g.nt * g.L, h->stream));
        gather_windows_kernel<<<blocks_for(g.n * g.L, 256), 256, 0, h->stream>>>(
            d_subject, g.loc, g.n, g.L, g.swin);
        CDTW_LAUNCH(h, "gather_windows_kernel");
        fill_kernel<<<blocks_for(g.n, 256), 256, 0, h->stream>>>(g.dD, g.n, 1.0f / k);
        CDTW_LAUNCH(h, "fill_kernel");
    }
    float* dloss = (float*)(base + o_loss);
    CDTW_CUDA(h, cudaStreamSynchronize(h->stream));
    // capture: main stream + nb branch streams
    cudaStream_t user = h->stream;
    cudaStream_t cs = h->own_stream;
    cl.s.resize(nb);
    cl.e.resize(2 * nb + 1);
    for (int b = 0; b < nb; ++b)
        CDTW_CUDA(h, cudaStreamCreateWithFlags(&cl.s[b], cudaStreamNonBlocking));
    for (auto& ev : cl.e) CDTW_CUDA(h, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    CDTW_CUDA(h, cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    int st = CDTW_OK;
    cudaEventRecord(cl.e[0], cs);
    for (int b = 0; b < nb; ++b) cudaStreamWaitEvent(cl.s[b], cl.e[0], 0);
    for (Group* gp : groups) {
        Group& g = *gp;
        const int b = g.branch;
        h->stream = cl.s[b];
        float* zq = (float*)(base + o_zq[b]);
        float* zs = (float*)(base + o_zs[b]);
        uint32_t* dirs = (uint32_t*)(base + o_dir[b]);
        uint32_t* rows = (uint32_t*)(g.path + (size_t)g.n * 32);
        uint32_t* cols = rows + (size_t)g.n * g.L;
        double* hdr = (double*)g.path;
        for (int s = 0; s <= steps && st == CDTW_OK; ++s) {
            broadcast_kernel<<<blocks_for(g.n * g.L, 256), 256, 0, h->stream>>>(g.tmpl, g.nt, k,
                                                                              g.L, g.qrep);
            st = launch_pair_znorm(h, g.qrep, g.swin, g.n, g.L, zq, zs, hdr);
            const bool last = s == steps;
            if (st == CDTW_OK)
                st = launch_pair_fwd(h, zq, zs, g.n, g.L, g.W, euclid, g.D, last ? nullptr : dirs,
                                     last ? nullptr : rows, last ? nullptr : cols);
            loss_kernel<<<g.nt, 32, 0, h->stream>>>(g.D, g.nt, k, g.dtid, dloss + (size_t)s * nt);
            if (last || st != CDTW_OK) break;
            st = launch_pair_bwd(h, g.qrep, g.swin, g.n, g.L, hdr, rows, cols, g.dD, euclid, g.dq,
                                 nullptr);
            const float c1 = 1.f - powf(kBeta1, (float)(s + 1));
            const float c2 = 1.f - powf(kBeta2, (float)(s + 1));
            adam_kernel<<<dim3(g.nt, (unsigned)div_up(g.L, 128)), 128, 0, h->stream>>>(
                g.dq, g.nt, k, g.L, g.tmpl, g.m, g.v, lr, c1, c2);
        }
    }
    for (int b = 0; b < nb; ++b) {
        cudaEventRecord(cl.e[1 + b], cl.s[b]);
        cudaStreamWaitEvent(cs, cl.e[1 + b], 0);
    }
    h->stream = cs;
    const cudaError_t ce = cudaStreamEndCapture(cs, &cl.g);
    h->stream = user;
    if (st != CDTW_OK) return st;
    if (ce != cudaSuccess) return check_cuda(h, ce, "cudaStreamEndCapture");
    CDTW_CUDA(h, cudaGraphInstantiate(&cl.x, cl.g, 0));
    // run after the caller's stream, copy the templates back
    CDTW_CUDA(h, cudaEventRecord(cl.e[nb + 1], user));
    CDTW_CUDA(h, cudaStreamWaitEvent(cs, cl.e[nb + 1], 0));
    CDTW_CUDA(h, cudaGraphLaunch(cl.x, cs));
    for (Group* gp : groups)
        for (int i = 0; i < gp->nt; ++i)
            CDTW_CUDA(h, cudaMemcpyAsync(d_templates + gp->toff[i], gp->tmpl + (size_t)i * gp->L,
                                         sizeof(float) * gp->L, cudaMemcpyDeviceToDevice, cs));
    if (losses)
        CDTW_CUDA(h, cudaMemcpyAsync(losses, dloss, sizeof(float) * (size_t)(steps + 1) * nt,
                                     cudaMemcpyDeviceToHost, cs));
    CDTW_CUDA(h, cudaStreamSynchronize(cs));
    return CDTW_OK;
}

// ---- refinement with the matches searched again at every step ---------------

namespace cdtw {

namespace {

// swin[(i k + j) L + e] = x[picks[i k2 + j] + e]: the first k picks of each
// of a group's templates, as the pair windows.
__global__ void gather_picks_kernel(const float* __restrict__ x, const int32_t* __restrict__ picks,
                                    int k, int k2, int64_t n, int L, float* __restrict__ out) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * L) return;
    const int64_t p = e / L;
    const int64_t i = p / k;
    const int64_t j = p - i * k;
    out[e] = __ldg(x + picks[i * k2 + j] + (e - p * L));
}

// A group of templates of equal (M, W) in the searching refinement: its
// pair buffers as in Group, plus the window statistics of length M and, per
// template, the picks of the last search (k2 windows, count and status).
struct SGroup {
    int L = 0, W = 0;
    std::vector<int> tids;
    std::vector<int64_t> toff;
    int nt = 0;
    int64_t n = 0;
    float *tmpl, *m, *v, *qrep, *swin, *D, *dq, *dD;
    double* mu;
    float* sigma;
    int32_t* picks;  // nt x k2
    float* pick_d;   // nt x k2
    int* cnt;        // nt x 2: picks found, status
    int* dtid;
    char* path;
    int branch = 0;
    double cost = 0.0;
};

}  // namespace

}  // namespace cdtw

extern "C" int cdtw_refine_templates_search(cdtw_handle h, const float* d_subject, int64_t N,
                                            float* d_templates, const int* Ms, const int* Ws,
                                            int nt, int k, int steps, float lr, int metric,
                                            float* losses, int64_t* locations) {
    if (!h) return CDTW_EINVAL;
    if (!d_subject || !d_templates || !Ms || !Ws || nt < 1 || k < 1 || steps < 0)
        return set_error(h, CDTW_EINVAL, "bad refinement arguments");
    if (metric != CDTW_EUCLIDEAN && metric != CDTW_MANHATTAN)
        return set_error(h, CDTW_EINVAL, "bad metric %d", metric);
    if (!(lr >= 0.f)) return set_error(h, CDTW_EINVAL, "bad learning rate");
    const bool euclid = metric == CDTW_EUCLIDEAN;
    const int k2 = 2 * k;
    std::map<std::pair<int, int>, SGroup> gm;
    int64_t off = 0;
    for (int t = 0; t < nt; ++t) {
        const int M = Ms[t];
        if (M < 11 || M > CDTW_MAX_QUERY || M > N)
            return set_error(h, CDTW_EINVAL, "template %d: length %d", t, M);
        if (N - M + 1 > (int64_t)INT32_MAX)
            return set_error(h, CDTW_EUNSUPPORTED, "too many windows");
        // k matches are guaranteed when the stream holds 2k seed segments
        if (div_up(N - M + 1, 2 * (int64_t)M) < k2)
            return set_error(h, CDTW_EINVAL,
                             "template %d: %lld samples hold fewer than 2k = %d segments of 2M",
                             t, (long long)N, k2);
        if (Ws[t] < 0) return set_error(h, CDTW_EINVAL, "template %d: negative band", t);
        const int W = std::min(Ws[t], M - 1);
        if (W > CDTW_PAIR_MAX_BAND)
            return set_error(h, CDTW_EUNSUPPORTED, "template %d: band %d exceeds %d", t, W,
                             CDTW_PAIR_MAX_BAND);
        SGroup& g = gm[{M, W}];
        g.L = M;
        g.W = W;
        g.tids.push_back(t);
        g.toff.push_back(off);
        off += M;
    }
    std::vector<SGroup*> groups;
    for (auto& kv : gm) groups.push_back(&kv.second);
    // longest-first assignment of the groups to the branches (search cells)
    const int nb = std::min<int>(kBranches, (int)groups.size());
    {
        for (SGroup* g : groups)
            g->cost = (double)g->tids.size() * g->L * (2.0 * g->W + 1.0);
        std::vector<SGroup*> ord = groups;
        std::sort(ord.begin(), ord.end(), [](SGroup* a, SGroup* b) { return a->cost > b->cost; });
        std::vector<double> load(nb, 0.0);
        for (SGroup* g : ord) {
            const int b = (int)(std::min_element(load.begin(), load.end()) - load.begin());
            g->branch = b;
            load[b] += g->cost;
        }
    }
    Slices c;
    std::vector<size_t> o_tm, o_m, o_v, o_q, o_s, o_D, o_dq, o_dD, o_tid, o_path, o_mu, o_sg,
        o_pk, o_pd, o_cnt;
    size_t zmax[kBranches] = {0}, dmax[kBranches] = {0}, pmax[kBranches] = {0},
           wmax[kBranches] = {0};
    for (SGroup* g : groups) {
        g->nt = (int)g->tids.size();
        g->n = (int64_t)g->nt * k;
        const int64_t Nw = N - g->L + 1;
        const size_t tl = (size_t)g->nt * g->L, pl = (size_t)g->n * g->L;
        o_tm.push_back(c.take<float>(tl));
        o_m.push_back(c.take<float>(tl));
        o_v.push_back(c.take<float>(tl));
        o_q.push_back(c.take<float>(pl));
        o_s.push_back(c.take<float>(pl));
        o_D.push_back(c.take<float>(g->n));
        o_dq.push_back(c.take<float>(pl));
        o_dD.push_back(c.take<float>(g->n));
        o_tid.push_back(c.take<int>(g->nt));
        o_path.push_back(c.take<char>(cdtw_pair_path_bytes(g->n, g->L)));
        o_mu.push_back(c.take<double>(Nw));
        o_sg.push_back(c.take<float>(Nw));
        o_pk.push_back(c.take<int32_t>((size_t)g->nt * k2));
        o_pd.push_back(c.take<float>((size_t)g->nt * k2));
        o_cnt.push_back(c.take<int>((size_t)g->nt * 2));
        const int b = g->branch;
        zmax[b] = std::max(zmax[b], pl);
        dmax[b] = std::max(dmax[b], (size_t)g->n * pair_dirs_words(g->L, g->W));
        pmax[b] = std::max(pmax[b], query_pack_layout(g->L, g->W, nullptr, nullptr));
        wmax[b] = std::max(wmax[b], topk_device_workspace_bytes(N, g->L, g->W, k2));
    }
    size_t o_zq[kBranches], o_zs[kBranches], o_dir[kBranches], o_pack[kBranches],
        o_ws[kBranches];
    for (int b = 0; b < nb; ++b) {
        o_zq[b] = c.take<float>(zmax[b]);
        o_zs[b] = c.take<float>(zmax[b]);
        o_dir[b] = c.take<uint32_t>(dmax[b]);
        o_pack[b] = c.take<char>(pmax[b]);
        o_ws[b] = c.take<char>(wmax[b]);
    }
    const size_t o_loss = c.take<float>((size_t)(steps + 1) * nt);
    CDTW_CUDA(h, cudaSetDevice(h->device));
    char* base = nullptr;
    CDTW_TRY(check_memory_limit(h, 0, c.off, "template refinement"));
    CDTW_CUDA(h, cudaMalloc(&base, c.off));
    struct Cleanup {
        char* p;
        std::vector<cudaStream_t> s;
        std::vector<cudaEvent_t> e;
        std::vector<cdtw_handle_s*> lanes;
        cudaGraph_t g = nullptr;
        cudaGraphExec_t x = nullptr;
        ~Cleanup() {
            if (x) cudaGraphExecDestroy(x);
            if (g) cudaGraphDestroy(g);
            for (auto st : s) cudaStreamSynchronize(st);
            for (cdtw_handle_s* l : lanes) {
                if (l->ring) cudaFree(l->ring);
                delete l;
            }
            for (auto ev : e) cudaEventDestroy(ev);
            for (auto st : s) cudaStreamDestroy(st);
            if (p) cudaFree(p);
        }
    } cl{base, {}, {}, {}};
    cudaStream_t user = h->stream;
    cudaStream_t cs = h->own_stream;
    cl.s.resize(nb);
    cl.e.resize(2 * nb + 1);
    for (int b = 0; b < nb; ++b)
        CDTW_CUDA(h, cudaStreamCreateWithFlags(&cl.s[b], cudaStreamNonBlocking));
    for (auto& ev : cl.e) CDTW_CUDA(h, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    // one search context per branch: its stream, query pack and work area
    for (int b = 0; b < nb; ++b) {
        cdtw_handle_s* l = new (std::nothrow) cdtw_handle_s();
        if (!l) return set_error(h, CDTW_ENOMEM, "refinement search context");
        cl.lanes.push_back(l);
        l->device = h->device;
        l->sm_count = h->sm_count;
        memcpy(l->band_variant, h->band_variant, sizeof(l->band_variant));
        l->stream = cl.s[b];
    }
    // set-up (outside the graph): templates in, statistics, moments 0
    for (size_t q = 0; q < groups.size(); ++q) {
        SGroup& g = *groups[q];
        g.tmpl = (float*)(base + o_tm[q]);
        g.m = (float*)(base + o_m[q]);
        g.v = (float*)(base + o_v[q]);
        g.qrep = (float*)(base + o_q[q]);
        g.swin = (float*)(base + o_s[q]);
        g.D = (float*)(base + o_D[q]);
        g.dq = (float*)(base + o_dq[q]);
        g.dD = (float*)(base + o_dD[q]);
        g.dtid = (int*)(base + o_tid[q]);
        g.path = base + o_path[q];
        g.mu = (double*)(base + o_mu[q]);
        g.sigma = (float*)(base + o_sg[q]);
        g.picks = (int32_t*)(base + o_pk[q]);
        g.pick_d = (float*)(base + o_pd[q]);
        g.cnt = (int*)(base + o_cnt[q]);
        CDTW_CUDA(h, cudaMemcpyAsync(g.dtid, g.tids.data(), sizeof(int) * g.nt,
                                     cudaMemcpyHostToDevice, h->stream));
        for (int i = 0; i < g.nt; ++i)
            CDTW_CUDA(h, cudaMemcpyAsync(g.tmpl + (size_t)i * g.L, d_templates + g.toff[i],
                                         sizeof(float) * g.L, cudaMemcpyDeviceToDevice,
                                         h->stream));
        CDTW_CUDA(h, cudaMemsetAsync(g.m, 0, sizeof(float) * g.nt * g.L, h->stream));
        CDTW_CUDA(h, cudaMemsetAsync(g.v, 0, sizeof(float) * g.nt * g.L, h->stream));
        CDTW_CUDA(h, cudaMemsetAsync(g.picks, 0, sizeof(int32_t) * g.nt * k2, h->stream));
        CDTW_CUDA(h, cudaMemsetAsync(g.cnt, 0, sizeof(int) * 2 * g.nt, h->stream));
        CDTW_TRY(launch_avg_std(h, d_subject, N, g.L, g.mu, g.sigma));
        fill_kernel<<<blocks_for(g.n, 256), 256, 0, h->stream>>>(g.dD, g.n, 1.0f / k);
        CDTW_LAUNCH(h, "fill_kernel");
    }
    float* dloss = (float*)(base + o_loss);
    CDTW_CUDA(h, cudaStreamSynchronize(h->stream));
    // the search of one template of a group (query pack from its current values)
    auto search = [&](SGroup& g, int i) -> int {
        cdtw_handle_s* l = cl.lanes[g.branch];
        query_pack_layout(g.L, g.W, &l->q, base + o_pack[g.branch]);
        l->has_query = true;
        int st = launch_prepare_query(l, g.tmpl + (size_t)i * g.L, g.L, g.W);
        int* cnt = g.cnt + 2 * i;
        int32_t* pk = g.picks + (size_t)i * k2;
        if (st == CDTW_OK)
            st = run_topk_device(l, d_subject, N, g.mu, g.sigma, euclid, k, k2,
                                 base + o_ws[g.branch], pk, cnt, pk, g.pick_d + (size_t)i * k2,
                                 cnt, cnt + 1);
        if (st != CDTW_OK) return set_error(h, st, "refinement search: %s", l->err);
        return CDTW_OK;
    };
    // eager search of every template: sizes any buffer a kernel family grows
    // on first use before the capture
    for (SGroup* gp : groups)
        for (int i = 0; i < gp->nt; ++i) CDTW_TRY(search(*gp, i));
    for (int b = 0; b < nb; ++b) CDTW_CUDA(h, cudaStreamSynchronize(cl.s[b]));
    for (SGroup* gp : groups)
        CDTW_CUDA(h, cudaMemsetAsync(gp->cnt, 0, sizeof(int) * 2 * gp->nt, h->stream));
    CDTW_CUDA(h, cudaStreamSynchronize(h->stream));
    // capture: every step of every group on its branch
    CDTW_CUDA(h, cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed));
    int st = CDTW_OK;
    cudaEventRecord(cl.e[0], cs);
    for (int b = 0; b < nb; ++b) cudaStreamWaitEvent(cl.s[b], cl.e[0], 0);
    for (int s = 0; s <= steps && st == CDTW_OK; ++s) {
        for (SGroup* gp : groups) {
            SGroup& g = *gp;
            const int b = g.branch;
            for (int i = 0; i < g.nt && st == CDTW_OK; ++i) st = search(g, i);
            if (st != CDTW_OK) break;
            h->stream = cl.s[b];
            float* zq = (float*)(base + o_zq[b]);
            float* zs = (float*)(base + o_zs[b]);
            uint32_t* dirs = (uint32_t*)(base + o_dir[b]);
            uint32_t* rows = (uint32_t*)(g.path + (size_t)g.n * 32);
            uint32_t* cols = rows + (size_t)g.n * g.L;
            double* hdr = (double*)g.path;
            gather_picks_kernel<<<blocks_for(g.n * g.L, 256), 256, 0, h->stream>>>(
                d_subject, g.picks, k, k2, g.n, g.L, g.swin);
            broadcast_kernel<<<blocks_for(g.n * g.L, 256), 256, 0, h->stream>>>(g.tmpl, g.nt, k,
                                                                              g.L, g.qrep);
            st = launch_pair_znorm(h, g.qrep, g.swin, g.n, g.L, zq, zs, hdr);
            const bool last = s == steps;
            if (st == CDTW_OK)
                st = launch_pair_fwd(h, zq, zs, g.n, g.L, g.W, euclid, g.D, last ? nullptr : dirs,
                                     last ? nullptr : rows, last ? nullptr : cols);
            loss_kernel<<<g.nt, 32, 0, h->stream>>>(g.D, g.nt, k, g.dtid, dloss + (size_t)s * nt);
            if (!last && st == CDTW_OK) {
                st = launch_pair_bwd(h, g.qrep, g.swin, g.n, g.L, hdr, rows, cols, g.dD, euclid,
                                     g.dq, nullptr);
                const float c1 = 1.f - powf(kBeta1, (float)(s + 1));
                const float c2 = 1.f - powf(kBeta2, (float)(s + 1));
                adam_kernel<<<dim3(g.nt, (unsigned)div_up(g.L, 128)), 128, 0, h->stream>>>(
                    g.dq, g.nt, k, g.L, g.tmpl, g.m, g.v, lr, c1, c2);
            }
            h->stream = user;
            if (st != CDTW_OK) break;
        }
    }
    for (int b = 0; b < nb; ++b) {
        cudaEventRecord(cl.e[1 + b], cl.s[b]);
        cudaStreamWaitEvent(cs, cl.e[1 + b], 0);
    }
    h->stream = cs;
    const cudaError_t ce = cudaStreamEndCapture(cs, &cl.g);
    h->stream = user;
    if (st != CDTW_OK) return st;
    if (ce != cudaSuccess) return check_cuda(h, ce, "cudaStreamEndCapture");
    CDTW_CUDA(h, cudaGraphInstantiate(&cl.x, cl.g, 0));
    CDTW_CUDA(h, cudaEventRecord(cl.e[nb + 1], user));
    CDTW_CUDA(h, cudaStreamWaitEvent(cs, cl.e[nb + 1], 0));
    CDTW_CUDA(h, cudaGraphLaunch(cl.x, cs));
    // results: templates, losses, the last step's matches
    for (SGroup* gp : groups)
        for (int i = 0; i < gp->nt; ++i)
            CDTW_CUDA(h, cudaMemcpyAsync(d_templates + gp->toff[i], gp->tmpl + (size_t)i * gp->L,
                                         sizeof(float) * gp->L, cudaMemcpyDeviceToDevice, cs));
    if (losses)
        CDTW_CUDA(h, cudaMemcpyAsync(losses, dloss, sizeof(float) * (size_t)(steps + 1) * nt,
                                     cudaMemcpyDeviceToHost, cs));
    std::vector<std::vector<int32_t>> hp(groups.size());
    std::vector<std::vector<int>> hc(groups.size());
    for (size_t q = 0; q < groups.size(); ++q) {
        hp[q].resize((size_t)groups[q]->nt * k2);
        hc[q].resize((size_t)groups[q]->nt * 2);
        CDTW_CUDA(h, cudaMemcpyAsync(hp[q].data(), groups[q]->picks, sizeof(int32_t) * hp[q].size(),
                                     cudaMemcpyDeviceToHost, cs));
        CDTW_CUDA(h, cudaMemcpyAsync(hc[q].data(), groups[q]->cnt, sizeof(int) * hc[q].size(),
                                     cudaMemcpyDeviceToHost, cs));
    }
    CDTW_CUDA(h, cudaStreamSynchronize(cs));
    for (size_t q = 0; q < groups.size(); ++q) {
        const SGroup& g = *groups[q];
        for (int i = 0; i < g.nt; ++i) {
            const int t = g.tids[i];
            if (hc[q][2 * i + 1] != 0)
                return set_error(h, CDTW_EUNSUPPORTED,
                                 "template %d: more windows under the top-k threshold than the "
                                 "hit list holds", t);
            if (hc[q][2 * i] < k)
                return set_error(h, CDTW_EUNSUPPORTED, "template %d: %d of %d matches found", t,
                                 hc[q][2 * i], k);
            if (locations)
                for (int j = 0; j < k; ++j)
                    locations[(int64_t)t * k + j] = hp[q][(size_t)i * k2 + j];
        }
    }
    return CDTW_OK;
}
