// selftest.cu -- the bounded-wait failure path, run on purpose.
//
// Every mbarrier wait of the step kernels gives up after tma::kWaitCycles,
// raises the call's error word and lets the kernel return, so that a load
// that never lands becomes a host-side error instead of a hung GPU.  The
// step kernels never reach that path in normal use; this entry drives it: one
// CTA waits, with a caller-given budget, on an mbarrier that no thread and no
// copy ever arrives at (nothing is in flight), and the host reads the error
// word exactly as the step loops' error check does.  With `arrive` set the
// CTA arrives first and the wait succeeds.
#include "tma.cuh"

namespace sweep {
namespace selftest {

enum { ERR_WAIT_SELFTEST = 9 };

// The error word of this entry (its own, so it never meets a step call's).
__device__ int g_selftest_err;

__global__ void wait_kernel(long long budget, int arrive)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        tma::mbar_init(&bar, 1);
        tma::fence_barrier_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (arrive) tma::mbar_arrive(&bar);
        tma::mbar_wait_for(&bar, 0, &g_selftest_err, ERR_WAIT_SELFTEST, budget);
    }
    __syncthreads();
}

}  // namespace selftest
}  // namespace sweep

using namespace sweep;

extern "C" int sweep_b200_wait_selftest(int64_t budget_cycles, int32_t arrive, void* stream, char* err,
                                        int32_t err_cap)
{
    return guarded(err, err_cap, [&] {
        SWEEP_REQUIRE(budget_cycles > 0 && budget_cycles <= tma::kWaitCycles,
                      "wait self-test: budget %lld cycles is outside (0, %lld]", (long long)budget_cycles,
                      (long long)tma::kWaitCycles);
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        const int zero = 0;
        SWEEP_CUDA(cudaMemcpyToSymbolAsync(selftest::g_selftest_err, &zero, sizeof(int), 0,
                                           cudaMemcpyHostToDevice, st));
        selftest::wait_kernel<<<1, 32, 0, st>>>((long long)budget_cycles, arrive ? 1 : 0);
        SWEEP_LAUNCH_CHECK();
        int h = 0;
        SWEEP_CUDA(cudaMemcpyFromSymbolAsync(&h, selftest::g_selftest_err, sizeof(int), 0,
                                             cudaMemcpyDeviceToHost, st));
        SWEEP_CUDA(cudaStreamSynchronize(st));
        SWEEP_REQUIRE(h == 0, "wait self-test: the mbarrier wait did not complete in time (code %d)", h);
    });
}
