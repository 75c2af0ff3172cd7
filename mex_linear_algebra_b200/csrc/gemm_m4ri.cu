// gemm_m4ri.cu -- GF(2) product by the Method of Four Russians on CUDA cores.
//
// Same result as the reference's mela_matmul_m4ri (src/mela_matmul_m4ri.c:
// 113-229): for every strip of 8 rows of B, a table of all 256 XOR
// combinations of those rows is built, and each row of C XORs the entry
// selected by its 8 bits of A.
//
// GPU organisation: a CTA owns a 1024-row x 1024-column block of C (8 warps
// x 128 rows; lane l holds 32-bit column l of the block for each of its
// rows, 128 accumulators).  Per stage of 32 values of k, the CTA builds 4
// tables (4 strips x 256 entries x 32 words = 128 KB of shared memory) in
// Gray-code order -- every entry costs one XOR and one store -- and then
// every row looks up its 4 entries: the table row is read by the 32 lanes
// at once (conflict-free 128-byte access), the row's 8-bit index is
// broadcast by a warp shuffle.
#include "mela_common.cuh"
#include "mela_internal.h"

namespace mela {

namespace {
__host__ __device__ constexpr int ctz_c(int x) { return (x & 1) ? 0 : 1 + ctz_c(x >> 1); }
constexpr int ROWS_PER_WARP = 128;
constexpr int WARPS = 8;
constexpr int CTA_ROWS = ROWS_PER_WARP * WARPS;  // 1024
constexpr int CTA_COLS32 = 32;                    // 32-bit columns per CTA (1024 bits)
constexpr int STRIPS = 4;                         // 8-row strips per stage
constexpr int TABLE_U32 = STRIPS * 256 * CTA_COLS32;
constexpr int SMEM_BYTES = TABLE_U32 * 4;         // 128 KB
}  // namespace

__global__ void __launch_bounds__(256, 1)
gemm_m4ri_kernel(const u64 *__restrict__ A, i64 lda, const u64 *__restrict__ B, i64 ldb,
                 u64 *__restrict__ C, i64 ldc, i64 m, i64 k, i64 n)
{
    extern __shared__ u32 T[];  // [STRIPS][256][32]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const i64 row0 = (i64)blockIdx.y * CTA_ROWS + warp * ROWS_PER_WARP;
    const i64 col32 = (i64)blockIdx.x * CTA_COLS32 + lane;  // this lane's 32-bit column
    const i64 ncol32 = 2 * words_of(n);
    const i64 nk32 = 2 * words_of(k);  // 32-bit words of K per row of A
    const bool col_ok = col32 < ncol32;

    // table-build role: strip (warp >> 1), Gray indices 128*(warp&1) .. +127
    const int bstrip = warp >> 1, bhalf = warp & 1;

    u32 acc[ROWS_PER_WARP];
#pragma unroll
    for (int r = 0; r < ROWS_PER_WARP; ++r) acc[r] = 0;

    const i64 nstages = (k + 31) / 32;

    auto load_b = [&](i64 st, u32 (&bv)[8]) {
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            const i64 kr = st * 32 + bstrip * 8 + b;
            bv[b] = (col_ok && kr < k) ? __ldg(reinterpret_cast<const u32 *>(B + kr * ldb) + col32) : 0u;
        }
    };
    auto load_a = [&](i64 st, u32 (&av)[4]) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const i64 r = row0 + j * 32 + lane;
            av[j] = (r < m && st < nk32) ? __ldg(reinterpret_cast<const u32 *>(A + r * lda) + st) : 0u;
        }
    };

    u32 bv[8], av[4];
    load_b(0, bv);
    load_a(0, av);

    for (i64 st = 0; st < nstages; ++st) {
        __syncthreads();  // previous stage's lookups are done with T
        {
            // Gray-code walk: entry g(i) = i ^ (i >> 1); entries 128..255 of the
            // walk are entries 0..127 with bits 7 and 6 flipped.
            u32 *Ts = T + bstrip * 256 * CTA_COLS32 + lane;
            u32 val = bhalf ? (bv[7] ^ bv[6]) : 0u;
            const u32 gflip = bhalf ? 192u : 0u;
            Ts[(0u ^ gflip) * CTA_COLS32] = val;
#pragma unroll
            for (int i = 1; i < 128; ++i) {
                val ^= bv[ctz_c(i)];
                const u32 g = ((u32)i ^ ((u32)i >> 1)) ^ gflip;
                Ts[g * CTA_COLS32] = val;
            }
        }
        __syncthreads();
        u32 cur_a[4] = {av[0], av[1], av[2], av[3]};
        if (st + 1 < nstages) {
            load_b(st + 1, bv);
            load_a(st + 1, av);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
#pragma unroll
            for (int r = 0; r < 32; ++r) {
                const u32 a = __shfl_sync(0xffffffffu, cur_a[j], r);
                u32 x = T[(0 * 256 + (a & 255u)) * CTA_COLS32 + lane];
                x ^= T[(1 * 256 + ((a >> 8) & 255u)) * CTA_COLS32 + lane];
                x ^= T[(2 * 256 + ((a >> 16) & 255u)) * CTA_COLS32 + lane];
                x ^= T[(3 * 256 + (a >> 24)) * CTA_COLS32 + lane];
                acc[j * 32 + r] ^= x;
            }
        }
    }

    if (col_ok) {
#pragma unroll
        for (int r = 0; r < ROWS_PER_WARP; ++r) {
            const i64 row = row0 + r;
            if (row < m) reinterpret_cast<u32 *>(C + row * ldc)[col32] = acc[r];
        }
    }
}

mela_status launch_gemm_m4ri(const u64 *A, i64 lda, const u64 *B, i64 ldb, u64 *C, i64 ldc, i64 m,
                             i64 k, i64 n, cudaStream_t s)
{
    if (m <= 0 || n <= 0) return MELA_OK;
    if (k <= 0) {
        MELA_CUDA_TRY(cudaMemset2DAsync(C, (size_t)ldc * 8, 0, (size_t)words_of(n) * 8, (size_t)m, s));
        return MELA_OK;
    }
    const i64 gx = (2 * words_of(n) + CTA_COLS32 - 1) / CTA_COLS32;
    const i64 gy = (m + CTA_ROWS - 1) / CTA_ROWS;
    if (gy > 65535) {
        set_error("gemm_m4ri: m too large for one launch");
        return MELA_ERR_UNSUPPORTED;
    }
    MELA_CUDA_TRY(cudaFuncSetAttribute(gemm_m4ri_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       SMEM_BYTES));
    gemm_m4ri_kernel<<<dim3((unsigned)gx, (unsigned)gy), 256, SMEM_BYTES, s>>>(A, lda, B, ldb, C, ldc,
                                                                                m, k, n);
    MELA_LAUNCH_CHECK("gemm_m4ri_kernel");
    return MELA_OK;
}

}  // namespace mela
