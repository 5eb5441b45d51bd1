// Dispatch of the register-band batched main pass (batch_reg.cuh): one
// kernel per band W <= 96, looked up at run time.
#include "batch_reg.cuh"

#include <algorithm>

namespace cdtw {

namespace {

struct BatchRegKernels {
    BatchRegKernel eu[kMaxRegW + 1];
    BatchRegKernel mh[kMaxRegW + 1];
    BatchRegKernels() {
        void** a = (void**)eu;
        void** b = (void**)mh;
        batch_reg_fill_part0(a, b);
        batch_reg_fill_part1(a, b);
        batch_reg_fill_part2(a, b);
        batch_reg_fill_part3(a, b);
        batch_reg_fill_part4(a, b);
        batch_reg_fill_part5(a, b);
    }
};

const BatchRegKernels& batch_reg_kernels() {
    static BatchRegKernels k;
    return k;
}

}  // namespace

int batch_reg_prepare(cdtw_handle h, int W, bool euclid, size_t smem, int* blocks) {
    if (W < 0 || W > kMaxRegW) return set_error(h, CDTW_EINVAL, "register band %d out of range", W);
    const void* k = (const void*)(euclid ? batch_reg_kernels().eu[W] : batch_reg_kernels().mh[W]);
    if (smem > 48 * 1024)
        CDTW_CUDA(h, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
    int per = 0;
    CDTW_CUDA(h, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, kBatchThreads, smem));
    *blocks = std::max(per, 1) * h->sm_count;
    return CDTW_OK;
}

int launch_batch_reg(cdtw_handle h, const BatchArgs& b, int W, bool euclid, size_t smem,
                     int blocks) {
    BatchRegKernel k = euclid ? batch_reg_kernels().eu[W] : batch_reg_kernels().mh[W];
    k<<<blocks, kBatchThreads, smem, h->stream>>>(b);
    CDTW_LAUNCH(h, "batch_reg_kernel");
    return CDTW_OK;
}

}  // namespace cdtw
