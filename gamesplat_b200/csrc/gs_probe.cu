// Failure-path probe (diagnostics): runs the library's bounded device waits
// against a word that nothing publishes, or an mbarrier whose transaction
// never arrives, with a caller-given poll limit, and records the error flag a
// frame would record.  This is how the timeout path is exercised without
// faulting or hanging a GPU: the wait runs out, the kernel returns, the host
// reads the flag and the context stays usable.
#include "gs_common.cuh"
#include "gs_internal.h"
#include "gs_tma.cuh"

namespace gs {

__global__ void wait_probe_kernel(const unsigned long long* status, FrameCounters* fc, uint32_t epoch, int which,
                                  uint32_t limit) {
    __shared__ __align__(8) uint64_t bar;
    if (which == 0) {
        // tile 1's look-back: tile 0's word carries another epoch, so it
        // reads as "not published yet" on every poll
        if (threadIdx.x < 32) {
            bool to = false;
            lookback_warp(status, 1, epoch, &to, limit);
            if (threadIdx.x == 0 && to) atomicOr(&fc->error_flags, kErrCullLookback);
        }
    } else {
        if (threadIdx.x == 0) {
            mbar_init(&bar, 1);
            mbar_fence_init();
        }
        __syncthreads();
        // 16 bytes are announced and no copy is issued: the phase never completes
        if (threadIdx.x == 0) mbar_arrive_expect_tx(&bar, 16u);
        __syncthreads();
        const bool ok = mbar_wait_bounded(&bar, 0u, limit);
        if (threadIdx.x == 0 && !ok) atomicOr(&fc->error_flags, kErrRasterWait);
    }
}

int launch_wait_probe(const unsigned long long* status, FrameCounters* fc, uint32_t epoch, int which, uint32_t limit,
                      cudaStream_t s) {
    wait_probe_kernel<<<1, 32, 0, s>>>(status, fc, epoch, which, limit);
    return 1;
}

}  // namespace gs
