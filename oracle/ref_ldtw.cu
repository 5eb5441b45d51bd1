// CPU runner of the reference's own LDTW host code -- TEST INFRASTRUCTURE ONLY.
//
// Compiles include/ldtw.cuh of the reference where it lies (the build recipe
// passes -I <reference>/include) and calls its host templates z_serial_ldtw
// (ldtw.cuh:74-127) and serial_ldtw (ldtw.cuh:19-71) for every window, as
// omp_z_stream_ldtw / omp_stream_ldtw do (ldtw.cuh:140-172).  Two shims let
// the header build with CUDA 12.9 without touching it:
//   * its include guard STATS_CUH is defined first, so stats.cuh (which pulls
//     in the vendored CUB that CUDA 12.9 no longer builds) is skipped; the
//     header's LDTW code uses nothing from it;
//   * `texture` (the texture-reference template CUDA 12 removed) is mapped to
//     an empty device-side stand-in, so the file-scope declarations of TS / TQ
//     (ldtw.cuh:11-12) parse; the GPU kernels that read them are templates
//     this runner never instantiates.
// The inputs of z_serial_ldtw are made as the reference's GPU-ldtw.cu makes
// them: the query z-normalised by znormalize (stats.cuh:8-28: float sums,
// population sigma), the window statistics by avg_std<double>
// (stats.cuh:30-52, :85-142: FP64 prefix sums of x and x^2, window means
// rounded to float, variance E[x^2] - mu^2 in float with the fused
// multiply-add nvcc makes of it, sigma = 1 where it is not positive).
//
//   ref_ldtw query.bin subject.bin M N W mode out.bin
//
// mode "z": z_serial_ldtw on the z-normalised query and windows; "raw":
// serial_ldtw on the query and windows as given.  Writes the N-M+1 float
// results to out.bin and prints the reference's determine_min line
// (ldtw.cuh:177-192).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <vector>

template <class T, int D, enum cudaTextureReadMode R>
struct RefTextureStandIn {};
template <class T, int D, enum cudaTextureReadMode R>
__device__ T tex1Dfetch(RefTextureStandIn<T, D, R>, int) {
    return T(0);
}
#define STATS_CUH
#define texture __device__ RefTextureStandIn
#include <ldtw.cuh>
#undef texture

// stats.cuh:8-28 (float accumulation, no contraction on the host)
static void ref_znormalize(float* x, int L) {
    float avg = 0, sd = 0;
    for (int i = 0; i < L; ++i) avg += x[i];
    avg /= L;
    for (int i = 0; i < L; ++i) sd += x[i] * x[i];
    sd = std::sqrt(sd / L - avg * avg);
    for (int i = 0; i < L; ++i) {
        x[i] -= avg;
        x[i] /= sd;
    }
}

// stats.cuh:30-52, :85-142 for one epoch (N <= 1e7 samples)
static void ref_avg_std(const float* s, int N, int M, float* avg, float* sd) {
    std::vector<double> p1(N + 1, 0.0), p2(N + 1, 0.0);
    for (int i = 0; i < N; ++i) {
        const double v = s[i];
        p1[i + 1] = p1[i] + v;
        p2[i + 1] = p2[i] + v * v;
    }
    for (int i = 0; i + M <= N; ++i) {
        const float mu = (float)((p1[i + M] - p1[i]) / M);
        const float ex2 = (float)((p2[i + M] - p2[i]) / M);
        const float var = std::fmaf(-mu, mu, ex2);
        avg[i] = mu;
        sd[i] = var > 0 ? std::sqrt(var) : 1.0f;
    }
}

static bool read_f32(const char* path, std::vector<float>& v, size_t n) {
    std::ifstream f(path, std::ios::binary | std::ios::in);
    if (!f) return false;
    v.resize(n);
    f.read(reinterpret_cast<char*>(v.data()), (std::streamsize)(sizeof(float) * n));
    return (size_t)f.gcount() == sizeof(float) * n;
}

int main(int argc, char* argv[]) {
    if (argc != 8) {
        std::fprintf(stderr, "usage: %s query.bin subject.bin M N W z|raw out.bin\n", argv[0]);
        return 2;
    }
    const int M = std::atoi(argv[3]), N = std::atoi(argv[4]), W = std::atoi(argv[5]);
    const bool zn = std::strcmp(argv[6], "z") == 0;
    std::vector<float> q, s;
    if (M < 1 || N < M || N > 10000000 || !read_f32(argv[1], q, M) || !read_f32(argv[2], s, N)) {
        std::fprintf(stderr, "bad arguments or input files\n");
        return 2;
    }
    const int nw = N - M + 1;
    std::vector<float> r(nw);
    if (zn) {
        ref_znormalize(q.data(), M);
        std::vector<float> avg(nw), sd(nw);
        ref_avg_std(s.data(), N, M, avg.data(), sd.data());
        omp_z_stream_ldtw<true>(q.data(), M, s.data(), N, avg.data(), sd.data(), r.data(), W);
    } else {
        omp_stream_ldtw<true>(q.data(), M, s.data(), N, r.data(), W);
    }
    std::ofstream o(argv[7], std::ios::binary);
    o.write(reinterpret_cast<const char*>(r.data()), (std::streamsize)(sizeof(float) * nw));
    determine_min<true>(r.data(), nw);
    return 0;
}
