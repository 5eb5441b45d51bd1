// UCR-DTW / UCR-DTW-BIN: drop-in replacements of the UCR Suite's DTW search
// tools that the reference ships beside its GPU drivers, running the search
// on the GPU through the streaming C ABI.
//
//   UCR-DTW      data.txt query.txt m R      (UCR Suite/UCR_DTW.cpp:381-427)
//   UCR-DTW-BIN  data.bin query.bin m R n    (UCR Suite/UCR_DTW_BIN.cpp:392-425)
//
// UCR-DTW reads whitespace-separated decimal numbers (fscanf("%lf"),
// UCR_DTW.cpp:511, :568-579); UCR-DTW-BIN raw float64 values (query m, data
// n).  R <= 1 is a band fraction (r = floor(R*m)), R > 1 the band itself
// (UCR_DTW.cpp:415-422).  The data file is read and pushed in pieces, as
// UCR reads it in EPOCH chunks, so its size is not bounded by device memory.
// The values are rounded to float32 for the device search (exact for data
// written from float32 samples).  Output lines are UCR's (UCR_DTW.cpp:714-727):
// Location, Distance, Data Scanned, Total Execution Time, and the pruning
// shares; "LB_Keogh" here is the forward and reverse LB_Keogh together (the
// device applies them in one pass), so the "LB_Keogh2" line reads 0.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <vector>

#include "cudadtw.h"

namespace {

// Reads up to `want` values into v (cleared first); false at the end.
struct Reader {
    FILE* f = nullptr;
    bool text = true;
    bool next(std::vector<float>& v, size_t want) {
        v.clear();
        if (text) {
            double d;
            while (v.size() < want && std::fscanf(f, "%lf", &d) == 1) v.push_back((float)d);
        } else {
            std::vector<double> buf(want);
            const size_t got = std::fread(buf.data(), sizeof(double), want, f);
            v.reserve(got);
            for (size_t i = 0; i < got; ++i) v.push_back((float)buf[i]);
        }
        return !v.empty();
    }
};

void usage(const char* self) {
#ifdef UCR_BINARY
    std::fprintf(stderr, "Usage: %s data.bin query.bin m R n\n", self);
#else
    std::fprintf(stderr, "Usage: %s data.txt query.txt m R\n", self);
#endif
}

}  // namespace

int main(int argc, char* argv[]) {
#ifdef UCR_BINARY
    const bool text = false;
    const int nargs = 6;
#else
    const bool text = true;
    const int nargs = 5;
#endif
    if (argc < nargs) {
        usage(argv[0]);
        return 1;
    }
    const int m = std::atoi(argv[3]);
    const double R = std::atof(argv[4]);
    const int r = R <= 1 ? (int)std::floor(R * m) : (int)std::floor(R);
    long long n_limit = -1;
#ifdef UCR_BINARY
    n_limit = std::atoll(argv[5]);
#endif
    Reader data, query;
    data.text = query.text = text;
    data.f = std::fopen(argv[1], text ? "r" : "rb");
    query.f = std::fopen(argv[2], text ? "r" : "rb");
    if (!data.f || !query.f) {
        std::fprintf(stderr, "ERROR: File not Found!!!\n");
        return 1;
    }
    const auto t1 = std::chrono::steady_clock::now();
    std::vector<float> q;
    query.next(q, (size_t)m);
    if ((int)q.size() != m || m < 11) {
        std::fprintf(stderr, "ERROR: need a query of m >= 11 values\n");
        return 1;
    }
    cdtw_handle h = nullptr;
    int st = cdtw_create(&h, 0);
    if (st == CDTW_OK) st = cdtw_stream_begin(h, q.data(), m, r, CDTW_EUCLIDEAN, 0);
    std::vector<float> chunk;
    long long read = 0;
    while (st == CDTW_OK && (n_limit < 0 || read < n_limit)) {
        size_t want = 1 << 20;
        if (n_limit >= 0) want = (size_t)std::min<long long>((long long)want, n_limit - read);
        if (!data.next(chunk, want)) break;
        read += (long long)chunk.size();
        st = cdtw_stream_push(h, chunk.data(), (int64_t)chunk.size());
    }
    int64_t loc = -1, scanned = 0;
    float dist = 0.f;
    if (st == CDTW_OK) st = cdtw_stream_end(h, &loc, &dist, &scanned);
    if (st != CDTW_OK) {
        std::fprintf(stderr, "ERROR: %s\n", h ? cdtw_last_error(h) : cdtw_status_string(st));
        if (h) cdtw_destroy(h);
        return 1;
    }
    int64_t c[3] = {0, 0, 0};
    cdtw_search_counts(h, c);
    cdtw_destroy(h);
    std::fclose(data.f);
    std::fclose(query.f);
    const auto t2 = std::chrono::steady_clock::now();
    const double secs = std::chrono::duration<double>(t2 - t1).count();
    const double i = (double)scanned;
    std::printf("\n");
    std::cout << "Location : " << loc << std::endl;
    std::cout << "Distance : " << dist << std::endl;
    std::cout << "Data Scanned : " << scanned << std::endl;
    std::cout << "Total Execution Time : " << secs << " sec" << std::endl;
    std::printf("\n");
    std::printf("Pruned by LB_Kim    : %6.2f%%\n", (double)(c[0] - c[1]) / i * 100);
    std::printf("Pruned by LB_Keogh  : %6.2f%%\n", (double)(c[1] - c[2]) / i * 100);
    std::printf("Pruned by LB_Keogh2 : %6.2f%%\n", 0.0);
    std::printf("DTW Calculation     : %6.2f%%\n", (double)c[2] / i * 100);
    return 0;
}
