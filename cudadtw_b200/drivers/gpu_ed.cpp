// GPU-ED: drop-in replacement of the reference driver GPU-ed.cu.
//
//   GPU-ED query.bin subject.bin M N
//
// Raw little-endian float64 files (query first, GPU-ed.cu:51-56), the same
// stdout lines (GPU-ed.cu:29-31, :67, :90; ed.cuh:322-324).  The
// z-normalised Euclidean search runs on the B200 through the C ABI
// (ed_search_host).  Short files and M > N are errors (exit status 1).
#include <chrono>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <vector>

#include "cudadtw.h"

static bool read_f64(const char* path, std::vector<double>& v, size_t n) {
    std::ifstream f(path, std::ios::binary | std::ios::in);
    if (!f) return false;
    v.resize(n);
    f.read(reinterpret_cast<char*>(v.data()), (std::streamsize)(sizeof(double) * n));
    return (size_t)f.gcount() == sizeof(double) * n;
}

int main(int argc, char* argv[]) {
    if (argc != 5) {
        std::cout << "call" << argv[0] << " query.bin subject.bin M N" << std::endl;
        return 1;
    }
    const int M = std::atoi(argv[3]);
    const long long N = std::atoll(argv[4]);
    std::cout << "\n= info =====================================" << std::endl;
    std::cout << "|Query| = " << M << "\t"
              << "|Subject| = " << N << "\t" << std::endl;
    if (M < 1 || N < M || M > CDTW_MAX_QUERY) {
        std::cerr << "ERROR: need 1 <= M <= N and M <= " << CDTW_MAX_QUERY << std::endl;
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
    std::vector<double> query, subject;
    if (!read_f64(argv[1], query, (size_t)M) || !read_f64(argv[2], subject, (size_t)N)) {
        std::cerr << "ERROR: could not read " << M << " / " << N << " float64 values" << std::endl;
        cdtw_destroy(h);
        return 1;
    }
    auto t1 = std::chrono::steady_clock::now();
    std::cout << "Miliseconds to load data: "
              << std::chrono::duration<double, std::milli>(t1 - t0).count() << std::endl;
    int64_t loc = -1;
    double dist = 0.0;
    t0 = std::chrono::steady_clock::now();
    st = ed_search_host(h, query.data(), M, subject.data(), N, &loc, &dist);
    t1 = std::chrono::steady_clock::now();
    if (st != CDTW_OK) {
        std::cerr << "ERROR: " << cdtw_last_error(h) << std::endl;
        cdtw_destroy(h);
        return 1;
    }
    std::cout << "\n= result ===================================" << std::endl;
    std::cout << "distance: " << dist << std::endl;
    std::cout << "location: " << loc << std::endl;
    std::cout << "Miliseconds to find best match: "
              << std::chrono::duration<double, std::milli>(t1 - t0).count() << std::endl;
    cdtw_destroy(h);
    return 0;
}
