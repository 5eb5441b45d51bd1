// GPU-LDTW: drop-in replacement of the reference driver GPU-ldtw.cu.
//
//   GPU-LDTW query.bin subject.bin M N P [--fp64 | --raw]
//
// Raw little-endian float32 files (query first), W = (int)(M * (P * 0.01))
// (GPU-ldtw.cu:412), the reference's GPU stdout lines (GPU-ldtw.cu:414,
// :439, :458, :470, :485-486, ldtw.cuh:189-191).  By default the path is
// computed in the reference's own FP32 arithmetic (ztsh2_ldtw with its
// statistics), so the reported index is the reference's; --fp64 takes FP64
// statistics and decisions instead; --raw runs the reference's tsh2_ldtw
// variant (GPU-ldtw.cu:87-88): the query z-normalised as the driver does,
// the windows raw.  The reference driver then re-runs the search on the host
// cores as a consistency check; this driver does not.
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <string>
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

// The driver's host z-normalisation of the query (znormalize,
// stats.cuh:8-28): float sums, population sigma, (x - avg) / std.
static void ref_znormalize(float* x, int L) {
    float avg = 0.f, sd = 0.f;
    for (int i = 0; i < L; ++i) avg += x[i];
    avg /= L;
    for (int i = 0; i < L; ++i) sd += x[i] * x[i];
    sd = std::sqrt(sd / L - avg * avg);
    for (int i = 0; i < L; ++i) {
        x[i] -= avg;
        x[i] /= sd;
    }
}

int main(int argc, char* argv[]) {
    const bool fp64 = argc == 7 && std::string(argv[6]) == "--fp64";
    const bool raw = argc == 7 && std::string(argv[6]) == "--raw";
    if (argc != 6 && !fp64 && !raw) {
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
    if (fp64) {
        st = ldtw_search_host(h, query.data(), M, subject.data(), N, W, CDTW_EUCLIDEAN, &loc,
                              &dist);
    } else {
        if (raw) ref_znormalize(query.data(), M);  // GPU-ldtw.cu:68 before the tsh2 line
        float d32 = 0.f;
        st = ldtw_ref_search_host(h, query.data(), M, subject.data(), N, W, CDTW_EUCLIDEAN,
                                  raw ? 0 : 1, &loc, &d32);
        dist = d32;
    }
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
