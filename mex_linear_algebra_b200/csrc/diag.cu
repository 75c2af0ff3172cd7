// diag.cu -- a diagnostic that drives the bounded-wait failure path.
//
// Every wait in the library's kernels (mbarrier phases of the tensor-core
// pipelines, the plain elimination's grid barrier) gives up after a limit,
// sets kErrWaitTimeout in the device error word, releases what it holds and
// returns; the host reports MELA_ERR_TIMEOUT.  This kernel makes such a wait
// run out on purpose, with a short limit, using the same wait helpers:
//   kind 0: a thread spins on a device flag that nothing ever sets;
//   kind 1: a CTA allocates tensor memory, then every thread waits on an
//           mbarrier that nothing arrives at; after the timeout the CTA
//           frees the tensor memory and returns.
// Nothing faults or traps and every wait ends, so the context stays usable.
#include "mela_common.cuh"
#include "mela_internal.h"
#include "mela_host.h"
#include "tc_ptx.cuh"

namespace mela {

namespace {
__device__ u32 g_never_set;  // stays zero: the flag kind 0 waits for
constexpr u32 kProbeTmemCols = 32;
}  // namespace

// out[0] = 1 when the wait ran out; out[1] = 1 once the tensor memory of
// kind 1 has been freed.
__global__ void __launch_bounds__(128, 1)
wait_timeout_probe_kernel(int kind, unsigned long long limit_ns, u32 *err, u32 *out)
{
    if (kind == 0) {
        if (threadIdx.x != 0) return;
        const volatile u32 *flag = &g_never_set;
        const unsigned long long t0 = global_ns();
        u32 timed_out = 0;
        while (*flag == 0) {
            if (global_ns() - t0 > limit_ns) {
                atomicOr(err, kErrWaitTimeout);
                timed_out = 1;
                break;
            }
        }
        out[0] = timed_out;
        return;
    }
    __shared__ __align__(8) u64 bar;
    __shared__ u32 tmem_slot;
    const int warp = threadIdx.x >> 5;
    if (warp == 0) {
        ptx::tmem_alloc(&tmem_slot, kProbeTmemCols);
        ptx::tmem_relinquish();
    }
    if (threadIdx.x == 0) {
        ptx::mbar_init(&bar, 1);
        ptx::fence_barrier_init();
    }
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    // phase 0 of a fresh barrier completes only after one arrival: none comes
    const bool ok = ptx::mbar_wait(&bar, 0, err, limit_ns);
    __syncthreads();
    if (threadIdx.x == 0) out[0] = ok ? 0u : 1u;
    if (warp == 0) {
        ptx::tc_fence_after();
        ptx::tmem_dealloc(tmem_slot, kProbeTmemCols);
    }
    __syncthreads();
    if (threadIdx.x == 0) out[1] = 1u;
}

}  // namespace mela

using namespace mela;

extern "C" mela_status mela_diag_wait_timeout(int32_t kind, uint64_t limit_ns, uint32_t *d_out, int32_t sync,
                                              void *stream)
{
    if ((kind != 0 && kind != 1) || limit_ns < 1000 || limit_ns > 1000000000ull || !d_out) {
        set_error("mela_diag_wait_timeout: kind 0 or 1, limit in [1 us, 1 s] and an output of two words");
        return MELA_ERR_INVALID;
    }
    u32 *err = device_error_word();
    if (!err) {
        set_error("device error word unavailable");
        return MELA_ERR_CUDA;
    }
    cudaStream_t s = (cudaStream_t)stream;
    wait_timeout_probe_kernel<<<1, 128, 0, s>>>(kind, (unsigned long long)limit_ns, err, d_out);
    MELA_LAUNCH_CHECK("wait_timeout_probe_kernel");
    if (!sync) return MELA_OK;
    return finish(s);
}
