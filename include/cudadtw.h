/*
 * cudadtw.h -- C ABI of the B200-native z-normalised subsequence search under a
 * Sakoe-Chiba band (the hot path of CUDA-DTW, gravitino/cudadtw).
 *
 * Every entry point returns an int status (CDTW_OK == 0) and never exits the
 * process; cdtw_last_error() gives the message of the last failure on a
 * handle.  Pointers named d_* are device pointers, h_* host pointers.  All
 * work runs on the handle's stream.  Device work buffers belong to the handle
 * (grow-only); callers own inputs and outputs.  One handle per host thread.
 *
 * Each declaration names the reference interface it replaces (file:line in
 * the reference project).  The reference keeps the query in __constant__
 * memory and the stream behind a texture reference set by the caller
 * (GPU-dtw.cu:46, :82-84); here both are per-handle state, so calls on
 * different handles are independent.
 */
#ifndef CUDADTW_H
#define CUDADTW_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cdtw_handle_s* cdtw_handle;

enum cdtw_status {
    CDTW_OK = 0,
    CDTW_EINVAL = 1,       /* bad argument (sizes, band, null pointer)            */
    CDTW_ENOMEM = 2,       /* device or pinned host allocation failed             */
    CDTW_ECUDA = 3,        /* a CUDA runtime call or kernel launch failed         */
    CDTW_ETIMEOUT = 4,     /* reserved: no entry point waits on the device for    */
                           /* another party, so none returns it                   */
    CDTW_EUNSUPPORTED = 5  /* valid request outside what this build implements     */
};

enum cdtw_metric {
    CDTW_EUCLIDEAN = 0,    /* squared difference cell cost (EUCLIDEAN, GPU-dtw.cu:7) */
    CDTW_MANHATTAN = 1     /* absolute difference cell cost (MANHATTAN, GPU-dtw.cu:8) */
};

enum cdtw_memloc { CDTW_HOST = 0, CDTW_DEVICE = 1 };

/* Largest query length accepted (the reference's MAXQUERYSIZE is 4096,
 * include/cdtw.cuh:8; 8192 for ED, include/ed.cuh:10). */
#define CDTW_MAX_QUERY 8192

/* ---- lifecycle ---------------------------------------------------------- */

/* Replaces cudaSetDevice(0)/cudaDeviceReset() + the global symbols of
 * GPU-dtw.cu:19-20.  Creates a handle bound to `device` and its own stream. */
int cdtw_create(cdtw_handle* out, int device);
int cdtw_destroy(cdtw_handle h);
/* Run all further work on `cuda_stream` (a cudaStream_t; NULL is the legacy
 * default stream, as in CUDA).  Until this is called the handle uses a
 * non-blocking stream of its own.  The stream argument of the reference
 * templates (cdtw.cuh:511, stats.cuh:116). */
int cdtw_set_stream(cdtw_handle h, void* cuda_stream);
const char* cdtw_last_error(cdtw_handle h);
const char* cdtw_status_string(int status);

/* Cap the device memory this handle holds (its grow-only work area, query
 * pack, strip rings, cached batched-search plan, and the per-call memory of
 * cdtw_refine_templates) at `bytes`; 0 removes the cap.  A call that would
 * need more fails with CDTW_ENOMEM before allocating, and the handle stays
 * usable for smaller calls.  No reference counterpart (prune_cdtw allocates
 * its temporaries unchecked and exits on failure, include/cdtw.cuh:521-525
 * with CUERR of include/cuda_def.cuh:6-8). */
int cdtw_set_memory_limit(cdtw_handle h, size_t bytes);

/* W = M*(P*0.01), truncated: GPU-dtw.cu:27 / GPU-ldtw.cu:412. */
int cdtw_band_from_percent(int M, int P);

/* ---- statistics ----------------------------------------------------------- */

/* Windowed mean and standard deviation of every length-M window of a float32
 * series: avg_std<double> (include/stats.cuh:115-142).  The mean is returned
 * in FP64, sigma in FP32; sigma = 1 where the variance is not positive
 * (stats.cuh:49-50).  Sums are FP64 with a per-warp shift, so level-shifted
 * series keep their variance (the reference's FP32 E[x^2]-mu^2 does not). */
int cdtw_avg_std(cdtw_handle h, const float* d_series, int64_t N, int M,
                 double* d_avg, float* d_std);

/* ---- query ---------------------------------------------------------------- */

/* z-normalise the query (FP64, population sigma; znormalize, stats.cuh:8-28)
 * and build its band envelope (envelope, bounds.cuh:13-64) into handle state.
 * Replaces the host z-norm + cudaMemcpyToSymbol(Czquery/Czlower/Czupper) of
 * GPU-dtw.cu:67-68, :82-84.  `query_loc` is CDTW_HOST or CDTW_DEVICE. */
int cdtw_set_query(cdtw_handle h, const float* query, int M, int W, int query_loc);

/* ---- banded DTW ------------------------------------------------------------ */

/* cDTW of the handle's query against listed windows of the subject:
 * gpu_cdtw (include/cdtw.cuh:450-487, kernels :164-431).  d_indices == NULL
 * means all N-M+1 windows in order (the raw, unpruned path of
 * tests/test_dtw.cu:98-109).  d_out[t] is the squared (Euclidean) or absolute
 * (Manhattan) cDTW of window d_indices[t] (or t).  d_avg/d_std come from
 * cdtw_avg_std with the same M. */
int cdtw_gpu_cdtw(cdtw_handle h, const float* d_subject, int64_t N,
                  const double* d_avg, const float* d_std,
                  const int32_t* d_indices, int64_t L, int metric, float* d_out);

/* Whole unpruned all-windows cDTW from host buffers: H2D of query and subject,
 * statistics, cDTW of every window, D2H of the N-M+1 results into h_out. */
int cdtw_all_windows_host(cdtw_handle h, const float* h_query, int M,
                          const float* h_subject, int64_t N, int W, int metric,
                          float* h_out);

/* ---- lower bounds ------------------------------------------------------------- */

/* LB_Kim of listed windows (all if d_indices == NULL): the reference's 5x5
 * front + 5x5 back unconstrained-DTW bound on the z-normalised window,
 * lb_kim (include/bounds.cuh:413-441, kernels :152-407).  Needs M >= 11
 * (bounds.cuh:418-422); returns CDTW_EINVAL otherwise. */
int cdtw_lb_kim(cdtw_handle h, const float* d_subject, int64_t N, const double* d_avg,
                const float* d_std, const int32_t* d_indices, int64_t L, int metric,
                float* d_out);

/* LB_Keogh of listed windows against the handle query's envelope, lb_keogh
 * (include/bounds.cuh:443-465, kernel :111-144) -> d_fwd; and the reverse
 * LB_Keogh of the query against the +-W envelope of the subject
 * (UCR Suite/UCR_DTW_BIN.cpp:262-282 with the envelope of :607) -> d_rev.
 * Either output may be NULL. */
int cdtw_lb_keogh(cdtw_handle h, const float* d_subject, int64_t N, const double* d_avg,
                  const float* d_std, const int32_t* d_indices, int64_t L, int metric,
                  float* d_fwd, float* d_rev);

/* ---- pruned search ------------------------------------------------------------- */

/* Best-matching window of the handle's query in the subject: prune_cdtw
 * (include/cdtw.cuh:510-592) + report_result (:493-508).  *location is the
 * window start (lowest index on ties, as UCR_DTW_BIN.cpp:682), *distance the
 * reference's printed "Distance:" (sqrt of the squared cDTW for the Euclidean
 * cost, the cDTW itself for Manhattan).  LB_Kim -> LB_Keogh / reverse
 * LB_Keogh -> early-abandoning cDTW, all on the device; one host sync at the
 * end.  Needs M >= 11. */
int cdtw_prune_cdtw(cdtw_handle h, const float* d_subject, int64_t N, const double* d_avg,
                    const float* d_std, int metric, int64_t* location, float* distance);

/* The k best pairwise non-overlapping windows of the handle's query: greedy
 * selection in (distance, window) order, a window overlapping (start within
 * M - 1 of) an accepted one is skipped.  locations[0..*found) / distances as
 * cdtw_prune_cdtw prints them, best first; *found < k only when the subject
 * holds fewer non-overlapping windows.  No reference counterpart (the
 * reference reports the single best match; UCR keeps one best-so-far).
 * Pruned like the search: LB_Kim, LB_Keogh and reverse LB_Keogh against a
 * threshold that provably bounds the k-th match (the 2k-th smallest cDTW of
 * pairwise non-overlapping seed windows).  Host-synchronous; needs M >= 11. */
int cdtw_topk(cdtw_handle h, const float* d_subject, int64_t N, const double* d_avg,
              const float* d_std, int metric, int k, int64_t* locations, float* distances,
              int* found);

/* cdtw_topk with every step on the device: the threshold by radix selection,
 * the windows under it collected by the early-abandoning search kernels, the
 * greedy selection in one thread block (the keys ordered only as far as it
 * consumes them).  The same picks as cdtw_topk; one host sync at the end.
 * The steps are those each iteration of cdtw_refine_templates_search runs
 * inside its CUDA graph.  CDTW_EUNSUPPORTED when more than min(N-M+1, 2^24)
 * windows fall under the threshold. */
int cdtw_topk_device(cdtw_handle h, const float* d_subject, int64_t N, const double* d_avg,
                     const float* d_std, int metric, int k, int64_t* locations,
                     float* distances, int* found);

/* The whole GPU-DTW search from host buffers (GPU-dtw.cu:59-90): H2D of the
 * subject and query, z-normalisation, statistics, pruned search. */
int cdtw_search_host(cdtw_handle h, const float* h_query, int M, const float* h_subject,
                     int64_t N, int W, int metric, int64_t* location, float* distance);

/* ---- search over a stream that arrives in pieces ------------------------------ */

/* The pruned search of cdtw_search_host over a subject that is pushed in
 * pieces of any size and never held whole on the device: the avg_std epochs
 * (include/stats.cuh:115-142) and the EPOCH loop of UCR_DTW_BIN.cpp:579-707,
 * which carries the last m-1 samples and the best-so-far from chunk to
 * chunk.  The device searches chunks of `chunk` samples (0: 2^23); each push
 * is copied straight into the current device chunk (from page-locked memory
 * in one copy, else through pinned staging buffers), the copies overlap the
 * search of the previous chunk, and every chunk's search starts from the
 * best distance of the chunks before it (kept on the device).  The caller
 * may reuse its buffer as soon as cdtw_stream_push returns.  The query (host, M >= 11 floats, band W) stays in
 * the handle until cdtw_stream_end; the handle must not run other searches
 * in between.  Windows are numbered from the first sample pushed (64-bit);
 * ties keep the earliest window, as UCR_DTW_BIN.cpp:682.  cdtw_stream_end
 * returns the best window, its printed distance (as cdtw_prune_cdtw) and the
 * number of samples scanned, and sets the stage counts and termination flag
 * (cdtw_search_counts / cdtw_search_flag) summed over the chunks.  The
 * device and pinned buffers stay with the handle after cdtw_stream_end and
 * serve the next stream when large enough (freed by cdtw_destroy); a begin
 * without an end before it drops the unfinished stream. */
int cdtw_stream_begin(cdtw_handle h, const float* h_query, int M, int W, int metric,
                      int64_t chunk);
int cdtw_stream_push(cdtw_handle h, const float* h_samples, int64_t n);
int cdtw_stream_end(cdtw_handle h, int64_t* location, float* distance, int64_t* scanned);

/* Stage counts of the last search on this handle: counts[0] windows,
 * counts[1] windows below the best-so-far after LB_Kim, counts[2] windows
 * that reached the cDTW stage.  No reference counterpart (UCR prints the
 * pruning percentages, UCR_DTW_BIN.cpp:738-741). */
int cdtw_search_counts(cdtw_handle h, int64_t* counts);

/* The line GPU-DTW prints after "Distance:" for the last search on this
 * handle: 1 when its best distance (squared for CDTW_EUCLIDEAN) lies below
 * the largest LB_Kim of any window, else 0.  prune_cdtw prints
 * (best_cdtw < max_kim) (include/cdtw.cuh:585), max_kim being LB_Kim at the
 * end of the ascending LB_Kim order it has searched (:541, :572); it stops
 * early only when best_cdtw < max_kim, and otherwise reaches the end of the
 * order, where max_kim is the largest LB_Kim of all, so the two agree. */
int cdtw_search_flag(cdtw_handle h, int* flag);

/* ---- batched search ------------------------------------------------------------- */

/* Best match of each of nq queries (lengths Ms[q], bands Ws[q]; the raw
 * float32 values concatenated in h_queries) in one device subject.  No
 * reference counterpart: the reference searches one query per process.
 *
 * rows == tiles == NULL (lengths up to CDTW_MAX_QUERY): every query runs the
 * cdtw_prune_cdtw pipeline, spread over 16 internal lanes (stream, query
 * pack, statistics, work area) that run concurrently, queries of one length
 * sharing their window statistics; the whole batch is one CUDA graph
 * (captured on the first call of a shape, replayed while the subject
 * pointer, N, lengths, bands and metric stay the same), one host sync per
 * call.  Results are bit-identical to cdtw_prune_cdtw's.
 *
 * With rows / tiles (lengths up to 4096): one graph of persistent kernels
 * that pull (query, stream-tile) work items from device queues: a seed pass
 * (tile statistics + LB_Kim), the cDTW of the seed windows, and a main pass
 * (statistics, LB_Kim, LB_Keogh, early-abandoning cDTW of the survivors).
 * rows[q] chooses the main-pass cDTW of the query's (length, band) bucket:
 * 0 = register band (one kernel per W <= 96), 1/2/4/8/16 = strips of that
 * many rows (W >= rows-1); tiles[q] is the windows per work item (a multiple
 * of 32 in [32, 4096]); either array may be NULL for the built-in choice
 * (register band up to W = 96, 16-row strips above, 1024-window tiles).
 *
 * Results as cdtw_prune_cdtw: window start (lowest on ties) and printed
 * distance. */
int cdtw_search_batched(cdtw_handle h, const float* d_subject, int64_t N,
                        const float* h_queries, const int* Ms, const int* Ws, int nq,
                        int metric, const int* rows, const int* tiles, int64_t* locations,
                        float* distances);

/* ---- GPU-ED: z-normalised Euclidean distance (float64) --------------------------- */

/* Squared z-normalised Euclidean distance of the query to every window,
 * d_out[w] = 2M - 2*corr(w)/sigma_w = sum_k (zq_k - z_k)^2, in FP64:
 * calculate_ed (include/ed.cuh:71-153) without the FFT and the argsort.
 * The raw float64 query is z-normalised on the device. */
int ed_all_windows(cdtw_handle h, const double* d_query, int M, const double* d_subject,
                   int64_t N, double* d_out);

/* The whole GPU-ED search from host buffers (GPU-ed.cu:51-82): *location is
 * the best window (lowest on ties), *distance = sqrt(min d^2), the
 * reference's "distance:" line (ed.cuh:323). */
int ed_search_host(cdtw_handle h, const double* h_query, int M, const double* h_subject,
                   int64_t N, int64_t* location, double* distance);

/* ---- GPU-LDTW: greedy local path in the band ---------------------------------- */

/* Cost of the greedy locally-optimal warping path of the handle's query
 * (cdtw_set_query, band W) against every window, FP64: ztsh2_ldtw
 * (include/ldtw.cuh:294-391), tie rule of ldtw.cuh:368-383. */
int ldtw_all_windows(cdtw_handle h, const float* d_subject, int64_t N, int metric,
                     double* d_out);

/* The whole GPU-LDTW search from host buffers (GPU-ldtw.cu:44-98): first
 * strict minimum (determine_min, ldtw.cuh:177-192); *distance = sqrt of the
 * path cost for the Euclidean cost. */
int ldtw_search_host(cdtw_handle h, const float* h_query, int M, const float* h_subject,
                     int64_t N, int W, int metric, int64_t* location, double* distance);

/* LDTW in the reference's own FP32 arithmetic, for drop-in index parity with
 * its GPU-LDTW.  znorm != 0: ztsh2_ldtw (include/ldtw.cuh:294-391) -- the
 * query z-normalised as GPU-ldtw.cu does on the host (znormalize,
 * stats.cuh:8-28, float sums), window statistics as avg_std<double>
 * (stats.cuh:30-52: FP64 window sums, variance E[x^2]-mu^2 in float),
 * samples (s-avg)/std, costs, comparisons and the path sum in float.
 * znorm == 0: tsh2_ldtw (ldtw.cuh:199-291) / serial_ldtw (:19-71), the query
 * as given to cdtw_set_query against the raw windows.  d_out: N-M+1 float
 * path costs (squared for CDTW_EUCLIDEAN).  Its decisions can differ from
 * ldtw_all_windows' FP64 ones on near-ties; on level-shifted series the
 * float variance loses precision exactly as the reference's does. */
int ldtw_ref_all_windows(cdtw_handle h, const float* d_subject, int64_t N, int metric, int znorm,
                         float* d_out);

/* The whole GPU-LDTW search in the reference's arithmetic from host buffers
 * (GPU-ldtw.cu:44-98 with ztsh2_ldtw, or its tsh2_ldtw line :87-88 when
 * znorm == 0): first strict minimum (determine_min, ldtw.cuh:177-192);
 * *distance = sqrt of the path cost for CDTW_EUCLIDEAN. */
int ldtw_ref_search_host(cdtw_handle h, const float* h_query, int M, const float* h_subject,
                         int64_t N, int W, int metric, int znorm, int64_t* location,
                         float* distance);

/* ---- fixed-scratch entry point ------------------------------------------------ */

/* Limits of cdtw_all_windows_noalloc and the size of its fixed device array. */
#define CDTW_NOALLOC_MAX_QUERY 4096
#define CDTW_NOALLOC_MAX_WINDOWS 1048576
#define CDTW_NOALLOC_SCRATCH_BYTES 12861696

/* All-windows cDTW that allocates nothing.  No counterpart in the reference.
 *
 * For callers that cannot let the library allocate device memory: hosts that
 * keep the device memory budget to themselves and lend the library only the
 * buffers of one call, or pipelines that cannot absorb the device-wide
 * synchronisation of cudaMalloc/cudaFree.  The handle API allocates (pinned
 * memory and a stream at cdtw_create, device work memory on first use); this
 * call takes no handle and calls no allocating routine.
 *
 * Computes the same as cdtw_set_query + cdtw_avg_std + cdtw_gpu_cdtw over all
 * N-M+1 windows: d_out[w] = squared (CDTW_EUCLIDEAN) or absolute
 * (CDTW_MANHATTAN) cDTW of the z-normalised raw query d_query (M floats, on
 * the device) against window w of d_subject.  Runs on `cuda_stream` (a
 * cudaStream_t; NULL = legacy default stream) on the current device.
 *
 * Working memory is one fixed __device__ array of CDTW_NOALLOC_SCRATCH_BYTES
 * (about 12.3 MiB) that every GPU loading the library keeps until exit.
 * Limits: M <= CDTW_NOALLOC_MAX_QUERY, N-M+1 <= CDTW_NOALLOC_MAX_WINDOWS,
 * band W <= 40 (after clamping W to M-1); larger requests return
 * CDTW_EUNSUPPORTED with the reason in errbuf (errlen bytes, may be NULL/0).
 * The first call on a device looks up the array's address on that device
 * (and again after the device's context was torn down and re-created, e.g.
 * by cudaDeviceReset); make that first call before any stream capture.  The
 * array's memory is reserved when the CUDA runtime loads this library's
 * device code, not by the call.  All calls on a device
 * share the one array: calls whose work overlaps on the GPU (different
 * streams, or host threads without ordering) race and corrupt each other's
 * results; order them on one stream. */
int cdtw_all_windows_noalloc(const float* d_query, int M, const float* d_subject, int64_t N,
                             int W, int metric, float* d_out, void* cuda_stream,
                             char* errbuf, int errlen);

/* ---- differentiable pairwise cDTW --------------------------------------------- */

#define CDTW_PAIR_ZNORM 1      /* z-normalise both series of every pair */
#define CDTW_PAIR_STORE_DIRS 2 /* path record from stored 2-bit directions */
#define CDTW_PAIR_RECOMPUTE 4  /* path record recomputed from checkpoints */
#define CDTW_PAIR_MAX_BAND 511 /* largest band W (after clamping W to L-1) */

/* Bytes of the path record of n pairs of length L: per pair the
 * z-normalisation constants (4 doubles) and the warping path as row and
 * column runs (2 x L 32-bit words).  8-byte aligned device memory. */
size_t cdtw_pair_path_bytes(int64_t n, int L);

/* Device work memory cdtw_pair_fwd takes from the handle's grow-only workspace
 * for n pairs: z-normalised copies of both series (flags & CDTW_PAIR_ZNORM)
 * and, when a path is recorded (with_path != 0), either 2 bits per band cell
 * of predecessor choices, padded to the lane layout, or (recomputation) two
 * anti-diagonals of the band every ~128 anti-diagonals.  The mode is that of
 * cdtw_pair_fwd without a memory limit on the handle.  0 for invalid sizes. */
size_t cdtw_pair_workspace_bytes(int64_t n, int L, int W, int flags, int with_path);

/* Path record modes of cdtw_pair_fwd (pairs whose record fits shared memory,
 * 2L-1 <= 512 and band W <= 15, always keep it there).  Stored directions:
 * the forward writes 2 bits per band cell to device scratch and walks them
 * back.  Recomputation from checkpoints: the forward keeps only two
 * anti-diagonals every ~128 (about 4x less scratch at L = 2048, W = 409),
 * and the walk recomputes each segment, last first, with its direction bits
 * in shared memory: the same path, bit for bit, for a second pass over the
 * band.  CDTW_PAIR_STORE_DIRS / CDTW_PAIR_RECOMPUTE force a mode; without
 * either, directions are stored unless their scratch would exceed 4 GiB (or
 * half the handle's memory limit).  No reference counterpart (the DP of
 * include/cdtw.cuh:24-88 returns distances only). */

/* 1 when the last cdtw_pair_fwd with a path record on this handle recomputed
 * from checkpoints, 0 when it stored direction bits.  No reference
 * counterpart. */
int cdtw_pair_last_mode(cdtw_handle h, int* recompute);

/* Banded cDTW of n pairs (d_q[p], d_s[p]), each L float32 samples, row-major
 * n x L on the device: d_D[p] = minimum over warping paths with |i-j| <= W of
 * the summed cell cost (squared difference for CDTW_EUCLIDEAN, absolute for
 * CDTW_MANHATTAN), the recurrence of include/cdtw.cuh:24-88 on two series.
 * flags & CDTW_PAIR_ZNORM normalises each series first (population sigma,
 * sigma = 1 when the variance is 0).  d_path (cdtw_pair_path_bytes, may be
 * NULL) receives the optimal path for cdtw_pair_bwd; the path is the
 * minimum-cost one under the rule: diagonal predecessor on ties, then
 * (i-1, j), then (i, j-1).  No reference counterpart.  1 <= L <= 8192. */
int cdtw_pair_fwd(cdtw_handle h, const float* d_q, const float* d_s, int64_t n, int L, int W,
                  int metric, int flags, float* d_D, void* d_path);

/* Gradient of sum_p d_dD[p] * D[p] with respect to the raw inputs (through the
 * z-normalisation when flags has CDTW_PAIR_ZNORM): the subgradient along the
 * path recorded by cdtw_pair_fwd, which must have run with the same inputs,
 * L, metric and flags.  d_dD may be NULL (all ones); d_dq or d_ds may be NULL
 * to skip that side.  Outputs n x L float32. */
int cdtw_pair_bwd(cdtw_handle h, const float* d_q, const float* d_s, int64_t n, int L,
                  int metric, int flags, const void* d_path, const float* d_dD, float* d_dq,
                  float* d_ds);

/* ---- template refinement ---------------------------------------------------------- */

/* Adam refinement of nt query templates against their matched windows (no
 * reference counterpart).  d_templates: the templates' raw float32 values
 * concatenated (sum of Ms floats, device), updated in place.  Template t
 * (length Ms[t], band Ws[t] <= CDTW_PAIR_MAX_BAND) is fitted to the k windows
 * of d_subject starting at locations[t*k .. t*k+k) (host array, e.g. from
 * cdtw_topk): loss_t = mean over its windows of the banded cDTW between the
 * z-normalised template and the z-normalised window (cdtw_pair_fwd with
 * CDTW_PAIR_ZNORM); each step takes the gradient through cdtw_pair_bwd and
 * applies Adam (learning rate lr, beta1 0.9, beta2 0.999, eps 1e-8) to the raw
 * template values.  All `steps` steps run as one CUDA graph.  losses (host,
 * may be NULL) receives (steps + 1) x nt values: row s = the losses before
 * step s, row `steps` = after the last step.  Host-synchronous; allocates its
 * working memory for the call. */
int cdtw_refine_templates(cdtw_handle h, const float* d_subject, int64_t N, float* d_templates,
                          const int* Ms, const int* Ws, int nt, const int64_t* locations, int k,
                          int steps, float lr, int metric, float* losses);

/* cdtw_refine_templates with the matches searched again at every step, all
 * inside the one CUDA graph: each step runs, per template, the device top-k
 * search of cdtw_topk_device (its candidate threshold also lowered by the
 * previous step's picks re-scored with the updated template), gathers the k
 * best non-overlapping windows as the pairs, then the pairwise forward,
 * backward and Adam update as cdtw_refine_templates.  Step `steps` only
 * searches and scores.  losses (host, (steps+1) x nt, may be NULL): mean
 * cDTW of each template to its matches of that step; locations (host,
 * nt x k, may be NULL): the matches of the last step, best first.  Needs
 * 11 <= M, W <= CDTW_PAIR_MAX_BAND and at least 2k segments of 2M windows
 * in the subject for every template (which guarantees k matches). */
int cdtw_refine_templates_search(cdtw_handle h, const float* d_subject, int64_t N,
                                 float* d_templates, const int* Ms, const int* Ws, int nt,
                                 int k, int steps, float lr, int metric, float* losses,
                                 int64_t* locations);

/* ---- kernel selection ----------------------------------------------------------- */

enum cdtw_variant {
    CDTW_VARIANT_AUTO = 0,      /* built-in rule: register band for W <= 96, lane groups up
                                   to W = 767, 16-row strips above                      */
    CDTW_VARIANT_REGISTER = 1,  /* one thread per window, the band in registers (W <= 96) */
    CDTW_VARIANT_STRIP16 = 2,   /* strips of 16 rows, boundary ring (W >= 15)            */
    CDTW_VARIANT_STRIP32 = 3,   /* strips of 32 rows, boundary ring (W >= 31)            */
    CDTW_VARIANT_LANE = 4       /* band spread over a lane group, two windows per group
                                   (27 <= W <= 767)                                     */
};

/* Kernel variant for bands w_lo..w_hi on this handle (what the autotuner,
 * cudadtw_b200/autotune.py, sets per (length, band) bucket).  A variant that
 * cannot run a band falls back to the built-in rule.  No reference
 * counterpart (gpu_cdtw's blockdtw flag chooses block vs thread kernels,
 * include/cdtw.cuh:450-487). */
int cdtw_set_band_variant(cdtw_handle h, int w_lo, int w_hi, int variant);

/* ---- measurement ------------------------------------------------------------ */

/* Issue-bound peak cell-update rate of the device (cells/s): the minimal cell
 * update (FADD, 3-input FMNMX, FFMA) on independent register chains.  The
 * roofline denominator of the cDTW kernels.  No reference counterpart (the
 * reference reports raw timings only, tests/test_dtw.cu:100-109). */
int cdtw_calibrate_cell_rate(cdtw_handle h, double* cells_per_second);

#ifdef __cplusplus
}
#endif

#endif /* CUDADTW_H */
