// Self-test of the bounded waits used by the tcgen05 kernels (no counterpart
// in the reference): a probe kernel waits on an mbarrier that nothing arrives
// on, so its wait runs out (umma::kWaitLimitCycles, about a second) and it
// reports through the device status word like the production kernels do.
#include "zg_internal.h"
#include "zg_umma.cuh"

namespace zg {

namespace {

__global__ void k_wait_probe(uint32_t *status) {
    using namespace umma;
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    // phase 0 never completes: the expected arrival never comes
    if (threadIdx.x == 0 && !mbar_wait(&bar, 0)) report_status(status, kStatusProbeTimeout);
}

}  // namespace

zg_status launch_wait_probe(zg_ctx *ctx, cudaStream_t s) {
    k_wait_probe<<<1, 32, 0, s>>>(ctx->status);
    ZG_CUDA(cudaGetLastError());
    ctx->launches++;
    return ZG_OK;
}

}  // namespace zg

extern "C" zg_status zg_debug_fail_allocation(uint32_t n) {
    zg::debug_fail_allocation(n);
    return ZG_OK;
}
