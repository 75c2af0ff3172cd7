// mela_common.cuh -- shared device/host helpers of the sm_100a GF(2) library.
//
// Packed layout used by every kernel: row-major uint64 words, bit j of row i
// in word i*ld + (j >> 6) at bit position (j & 63) -- the reference library's
// own convention (src/mela_matmul_gf2.c:33-36).  Bits at columns >= n of the
// last word of a row are zero on every packed buffer this library writes.
#pragma once

#include <cstdint>
#include <cstddef>
#include <cuda_runtime.h>

#include "../../include/mela.h"

namespace mela {

using u64 = unsigned long long;
using u32 = unsigned int;
using i64 = long long;

constexpr int kWordBits = 64;
__host__ __device__ inline i64 words_of(i64 n) { return (n + 63) >> 6; }

// ---------------------------------------------------------------- errors
// Thread-local detail message of the last failure (host side).
void set_error(const char *fmt, ...);
mela_status cuda_status(cudaError_t e, const char *what);

#define MELA_CUDA_TRY(expr)                                        \
    do {                                                           \
        cudaError_t _e = (expr);                                   \
        if (_e != cudaSuccess) return ::mela::cuda_status(_e, #expr); \
    } while (0)

#define MELA_LAUNCH_CHECK(what)                                    \
    do {                                                           \
        cudaError_t _e = cudaGetLastError();                       \
        if (_e != cudaSuccess) return ::mela::cuda_status(_e, what); \
    } while (0)

// Device-side error word.  Kernels whose waits can run out set a bit here
// instead of trapping; the host reads it with mela_device_error_flags().
enum : u32 {
    kErrWaitTimeout = 1u << 0,   // an mbarrier / flag wait ran past its limit
    kErrBadArgument = 1u << 1,   // a kernel-side bounds check rejected its input
};
u32 *device_error_word();  // per-device __device__ word (address on current device)

// Timeout for every bounded device-side wait: about two seconds.
constexpr unsigned long long kWaitLimitNs = 2000000000ull;

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// ---------------------------------------------------------------- launch sizing
int sm_count();  // multiprocessors of the current device (cached per device)

// A grid's y and z extents are limited to 65535 blocks: larger shapes are
// refused up front (MELA_ERR_UNSUPPORTED) instead of failing at launch.
inline mela_status check_grid_yz(i64 y, i64 z, const char *what)
{
    if (y > 65535 || z > 65535) {
        set_error("%s: shape needs a grid of %lld x %lld blocks in y and z (limit 65535)", what, y, z);
        return MELA_ERR_UNSUPPORTED;
    }
    return MELA_OK;
}

// 32 x 32 bit transpose across a warp: lane r passes row r (bit c = column
// c); lane c gets column c (bit r = row r).  Five rounds of shuffle
// butterflies: at round s the lanes with bit s clear trade their columns
// c + s (bit s of c set) for the columns c of lane r + s.
__device__ __forceinline__ unsigned transpose32_warp(unsigned v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int sh = 16; sh >= 1; sh >>= 1) {
        const unsigned m = sh == 16 ? 0x0000FFFFu : sh == 8 ? 0x00FF00FFu : sh == 4 ? 0x0F0F0F0Fu
                         : sh == 2  ? 0x33333333u : 0x55555555u;
        const unsigned o = __shfl_xor_sync(0xffffffffu, v, sh);
        v = (lane & sh) ? ((v & ~m) | ((o >> sh) & m)) : ((v & m) | ((o & m) << sh));
    }
    return v;
}

}  // namespace mela
