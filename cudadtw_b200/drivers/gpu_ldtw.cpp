// GPU-LDTW: drop-in replacement of the reference driver GPU-ldtw.cu.
//
//   GPU-LDTW query.bin subject.bin M N P
//
// Raw little-endian float32 files (query first), W = (int)(M * (P * 0.01))
// (GPU-ldtw.cu:412), the reference's GPU stdout lines (GPU-ldtw.cu:414,
// :439, :458, :470, :485-486, ldtw.cuh:189-191).  The reference driver then
// re-runs the search on the host cores as a consistency check; this driver
// does not (the CPU restatement lives in the test oracle).
#include <chrono>
#include <cstdlib>
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
    if (argc != 6) {
        std::cout << "call" << argv[0] << " query.bin subject.bin M N P" << std::endl;
        return 1;
    }
    const int M = std::atoi(argv[3]);
    const long long N = std::atoll(argv[4]);
    const int W = cdtw_band_from_percent(M, std::atoi(argv[5]));
    std::cout << " M " << M << " N " << N << " W " << W << std::endl;
    if (M < 1 || N < M) {
        std::cerr << "ERROR: need 1 <= M <= N" << std::endl;
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
    std::cout << "\n= aligning==================================" << std::endl;
    int64_t loc = -1;
    double dist = 0.0;
    t0 = std::chrono::steady_clock::now();
    st = ldtw_search_host(h, query.data(), M, subject.data(), N, W, CDTW_EUCLIDEAN, &loc, &dist);
    t1 = std::chrono::steady_clock::now();
    if (st != CDTW_OK) {
        std::cerr << "ERROR: " << cdtw_last_error(h) << std::endl;
        cdtw_destroy(h);
        return 1;
    }
    std::cout << "Miliseconds to find best alignment on the GPU: "
              << std::chrono::duration<double, std::milli>(t1 - t0).count() << std::endl;
    std::cout << "best alignment found at index " << loc << " with distance " << dist
              << std::endl
              << std::endl;
    cdtw_destroy(h);
    return 0;
}
