// GPU-DTW: drop-in replacement of the reference driver GPU-dtw.cu.
//
//   GPU-DTW query.bin subject.bin M N P [--json]
//
// Same argv, raw little-endian float32 files (query first), band
// W = (int)(M * (P * 0.01)) (GPU-dtw.cu:27) and the same stdout lines
// (GPU-dtw.cu:29-32, :74, :96; cdtw.cuh:506-507, :585), so the reference's
// bench scripts parse it unchanged.  The search runs on the B200 through the
// C ABI (cdtw_search_host).  The "1" line is the reference's early-termination
// flag; this search always examines every window it cannot prune, so it is
// always 1.  Unlike the reference, short files, M > N and M < 11 are errors
// (exit status 1) instead of reading uninitialised memory.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <vector>

#include "cudadtw.h"

static bool read_f32(const char* path, std::vector<float>& v, size_t n) {
    std::ifstream f(path, std::ios::binary | std::ios::in);
    if (!f) return false;
    v.resize(n);
    f.read(reinterpret_cast<char*>(v.data()), (std::streamsize)(sizeof(float) * n));
    return (size_t)f.gcount() == sizeof(float) * n;
}

int main(int argc, char* argv[]) {
    const bool json = argc == 7 && std::strcmp(argv[6], "--json") == 0;
    if (argc != 6 && !json) {
        std::cout << "call" << argv[0] << " query.bin subject.bin M N P" << std::endl;
        return 1;
    }
    const int M = std::atoi(argv[3]);
    const long long N = std::atoll(argv[4]);
    const int W = cdtw_band_from_percent(M, std::atoi(argv[5]));

    std::cout << "\n= info =====================================" << std::endl;
    std::cout << "|Query| = " << M << "\t"
              << "|Subject| = " << N << "\t"
              << "window = " << W << std::endl;
    if (M < 11 || N < M) {
        std::cerr << "ERROR: need 11 <= M <= N" << std::endl;
        return 1;
    }
    cdtw_handle h = nullptr;
    int st = cdtw_create(&h, 0);
    if (st != CDTW_OK) {
        std::cerr << "ERROR: cdtw_create: " << cdtw_status_string(st) << std::endl;
        return 1;
    }
    std::cout << "\n= loading data =============================" << std::endl;
    auto t0 = std::chrono::steady_clock::now();
    std::vector<float> query, subject;
    if (!read_f32(argv[1], query, (size_t)M) || !read_f32(argv[2], subject, (size_t)N)) {
        std::cerr << "ERROR: could not read " << M << " / " << N << " float32 values" << std::endl;
        cdtw_destroy(h);
        return 1;
    }
    auto t1 = std::chrono::steady_clock::now();
    std::cout << "Miliseconds to load data: "
              << std::chrono::duration<double, std::milli>(t1 - t0).count() << std::endl;
    std::cout << "\n= pruning ==================================" << std::endl;
    int64_t loc = -1;
    float dist = 0.f;
    t0 = std::chrono::steady_clock::now();
    st = cdtw_search_host(h, query.data(), M, subject.data(), N, W, CDTW_EUCLIDEAN, &loc, &dist);
    t1 = std::chrono::steady_clock::now();
    if (st != CDTW_OK) {
        std::cerr << "ERROR: " << cdtw_last_error(h) << std::endl;
        cdtw_destroy(h);
        return 1;
    }
    const double ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    std::cout << "Location: " << loc << std::endl;
    std::cout << "Distance: " << dist << std::endl;
    int flag = 0;
    cdtw_search_flag(h, &flag);  // (best < largest LB_Kim), include/cdtw.cuh:585
    std::cout << flag << std::endl;
    std::cout << "Miliseconds to find best match: " << ms << std::endl;
    if (json) {
        int64_t c[3];
        cdtw_search_counts(h, c);
        std::printf("{\"location\": %lld, \"distance\": %.9g, \"ms\": %.4f, \"M\": %d, \"N\": %lld, "
                    "\"W\": %d, \"windows\": %lld, \"after_lb_kim\": %lld, \"dtw\": %lld}\n",
                    (long long)loc, dist, ms, M, N, W, (long long)c[0], (long long)c[1],
                    (long long)c[2]);
    }
    cdtw_destroy(h);
    return 0;
}
