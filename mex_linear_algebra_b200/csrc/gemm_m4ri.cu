// gemm_m4ri.cu -- GF(2) product by the Method of Four Russians on CUDA cores.
//
// Same result as the reference's mela_matmul_m4ri (src/mela_matmul_m4ri.c:
// 113-229): for every strip of 8 rows of B, a table of all 256 XOR
// combinations of those rows is built, and each row of C XORs the entry
// selected by its 8 bits of A.
//
// GPU organisation: a CTA owns a 512-row x 2048-column block of C; lane l of
// every warp holds 64-bit column word l of the block; 16 warps own 32 rows
// each (the default tile), or 8 warps 64 rows each (tile 1: fewer, fatter
// warps).  K advances 16 bits per stage: the warps build the stage's two
// tables (2 strips x 256 entries x 32 words = 128 KB of shared memory), an
// equal share of the entries each in Gray-code order --
// one 64-bit XOR and one store per entry --, then every row looks up its two
// entries: the 32 lanes read one entry's 256 contiguous bytes (two
// conflict-free wavefronts), the row's 16 index bits come from the lane that
// holds the row's word of A by one shuffle.  Per 16 x 2048 bit-products of a
// row: two table reads and two XORs, against 32 AND+XOR word operations in
// the plain form.
//
// The 16 rows of B a stage needs (32 words each) are staged by TMA: one 2-D
// tile load per stage into a double-buffered 4 KB tile, issued one stage
// ahead by one thread and counted on an mbarrier (bounded wait), zeros past
// the matrix edges.  The table builders read their 8 rows from that tile.
// Where TMA cannot address B (a row pitch that is not a multiple of 16 bytes,
// or an unaligned base) the rows are read with ordinary loads instead.
#include "mela_common.cuh"
#include "mela_internal.h"
#include "tc_ptx.cuh"

#include <cstring>

namespace mela {

namespace {
__host__ __device__ constexpr int ctz_c(int x) { return (x & 1) ? 0 : 1 + ctz_c(x >> 1); }
constexpr int M4_CTA_ROWS = 512;                            // rows of C per CTA (8 or 16 warps)
constexpr int M4_CTA_WORDS = 32;                            // 64-bit column words per CTA (2048 columns)
constexpr int M4_STRIPS = 2;                                // 8-row strips of B per stage (16 bits of K)
constexpr int M4_SMEM_BYTES = M4_STRIPS * 256 * M4_CTA_WORDS * 8;  // 128 KB

// Steps J.. of an E-entry Gray-code walk from position i0 (a multiple of E):
// store the running XOR at entry g(i) = i ^ (i >> 1), then add the B row
// whose bit flips next (bit ctz(i + 1) = ctz(J + 1), a constant here).
template <int J, int E>
__device__ __forceinline__ void gray_walk(u64 *Ts, int i0, u64 &val, const u64 (&bv)[8])
{
    if constexpr (J < E) {
        const int i = i0 + J;
        Ts[(i ^ (i >> 1)) * M4_CTA_WORDS] = val;
        if constexpr (J < E - 1) val ^= bv[ctz_c(J + 1)];
        gray_walk<J + 1, E>(Ts, i0, val, bv);
    }
}
}  // namespace

constexpr int M4_BTILE_WORDS = 16 * M4_CTA_WORDS;  // one stage's rows of B (4 KB)

template <int WARPS, bool kTma>
__global__ void __launch_bounds__(WARPS * 32, 1)
gemm_m4ri_kernel(const u64 *__restrict__ A, i64 lda, const u64 *__restrict__ B, i64 ldb,
                 u64 *__restrict__ C, i64 ldc, i64 m, i64 k, i64 n, const __grid_constant__ CUtensorMap bmap,
                 u32 *err)
{
    extern __shared__ __align__(128) u64 T[];  // [M4_STRIPS][256][32], then [2][16][32] rows of B
    u64 *Bt = T + M4_STRIPS * 256 * M4_CTA_WORDS;
    __shared__ __align__(8) u64 bfull[2];
    constexpr int M4_ROWS_PER_WARP = M4_CTA_ROWS / WARPS;  // 64 or 32
    constexpr int H = M4_ROWS_PER_WARP / 32;                 // rows per lane held for A
    constexpr int WALK = 2 * 256 / WARPS;                     // Gray-walk entries per warp
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const i64 row0 = (i64)blockIdx.y * M4_CTA_ROWS + warp * M4_ROWS_PER_WARP;
    const i64 cw = (i64)blockIdx.x * M4_CTA_WORDS + lane;  // this lane's column word
    const i64 ncw = words_of(n), kw = words_of(k);
    const bool col_ok = cw < ncw;

    // table-build role: strip bstrip, Gray-walk positions WALK*bq .. WALK*bq+WALK-1
    const int bstrip = warp / (WARPS / 2), bq = warp % (WARPS / 2);

    u64 acc[M4_ROWS_PER_WARP];
#pragma unroll
    for (int r = 0; r < M4_ROWS_PER_WARP; ++r) acc[r] = 0;

    const i64 nstages = (k + 15) / 16;

    // B: the 8 rows of this warp's strip in stage st, this lane's word
    auto load_b = [&](i64 st, u64 (&bv)[8]) {
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            const i64 kr = st * 16 + bstrip * 8 + b;
            bv[b] = (col_ok && kr < k) ? __ldg(B + kr * ldb + cw) : 0ull;
        }
    };
    // TMA: rows 16*st .. 16*st+15, words cw0 .. cw0+31 into tile buffer st & 1
    const int cw0 = (int)((i64)blockIdx.x * M4_CTA_WORDS);
    auto issue_b = [&](i64 st) {
        const int buf = (int)(st & 1);
        ptx::mbar_arrive_expect_tx(&bfull[buf], M4_BTILE_WORDS * 8);
        ptx::tma_load_2d(Bt + buf * M4_BTILE_WORDS, &bmap, &bfull[buf], cw0, (int)(st * 16));
    };
    // A: word w of K for rows row0 + 32h + lane
    auto load_a = [&](i64 w, u64 (&av)[H]) {
#pragma unroll
        for (int h = 0; h < H; ++h) {
            const i64 r = row0 + 32 * h + lane;
            av[h] = (r < m && w < kw) ? __ldg(A + r * lda + w) : 0ull;
        }
    };

    u64 bv[8], av[H], av_next[H];
    if constexpr (kTma) {
        if (threadIdx.x == 0) {
            ptx::prefetch_tmap(&bmap);
            ptx::mbar_init(&bfull[0], 1);
            ptx::mbar_init(&bfull[1], 1);
            ptx::fence_barrier_init();
            issue_b(0);
        }
        __syncthreads();
    } else {
        load_b(0, bv);
    }
    load_a(0, av);
    load_a(1, av_next);

    for (i64 st = 0; st < nstages; ++st) {
        const int sub = (int)(st & 3);  // 16-bit slice of the current A word
        if constexpr (kTma) {
            // this stage's rows of B have landed (every thread waits, bounded);
            // the barrier after it also ends the previous stage's lookups
            const bool ok = ptx::mbar_wait(&bfull[st & 1], (u32)((st >> 1) & 1), err);
            if (__syncthreads_or(!ok)) {
                // a wait ran out (timeout bit set): give the copy in flight one
                // more bounded wait, then leave without writing C
                if (threadIdx.x == 0) ptx::mbar_wait(&bfull[st & 1], (u32)((st >> 1) & 1), nullptr);
                return;
            }
            // the other tile was last read by the previous stage's builders
            if (threadIdx.x == 0 && st + 1 < nstages) issue_b(st + 1);
            const u64 *rows = Bt + (int)(st & 1) * M4_BTILE_WORDS + bstrip * 8 * M4_CTA_WORDS + lane;
#pragma unroll
            for (int b = 0; b < 8; ++b) bv[b] = rows[b * M4_CTA_WORDS];
        } else {
            __syncthreads();  // the previous stage's lookups are done with T
        }
        {
            u64 *Ts = T + (size_t)bstrip * 256 * M4_CTA_WORDS + lane;
            const int i0 = WALK * bq;
            const int g0 = i0 ^ (i0 >> 1);
            u64 val = 0;
#pragma unroll
            for (int b = 0; b < 8; ++b)
                if ((g0 >> b) & 1) val ^= bv[b];
            gray_walk<0, WALK>(Ts, i0, val, bv);
        }
        __syncthreads();
        // the 16 bits of K of this stage for rows 32h + lane
        u32 ix[H];
#pragma unroll
        for (int h = 0; h < H; ++h) ix[h] = (u32)(av[h] >> (16 * sub)) & 0xffffu;
        if (st + 1 < nstages) {
            if constexpr (!kTma) load_b(st + 1, bv);
            if (sub == 3) {
#pragma unroll
                for (int h = 0; h < H; ++h) av[h] = av_next[h];
                load_a((st + 1) / 4 + 1, av_next);
            }
        }
        const u64 *T0 = T + lane;
        const u64 *T1 = T + 256 * M4_CTA_WORDS + lane;
#pragma unroll
        for (int r = 0; r < M4_ROWS_PER_WARP; ++r) {
            const u32 x = __shfl_sync(0xffffffffu, ix[r / 32], r & 31);
            acc[r] ^= T0[(x & 255u) * M4_CTA_WORDS] ^ T1[(x >> 8) * M4_CTA_WORDS];
        }
    }

    if (col_ok) {
#pragma unroll
        for (int r = 0; r < M4_ROWS_PER_WARP; ++r) {
            const i64 row = row0 + r;
            if (row < m) C[row * ldc + cw] = acc[r];
        }
    }
}

mela_status launch_gemm_m4ri(const u64 *A, i64 lda, const u64 *B, i64 ldb, u64 *C, i64 ldc, i64 m,
                             i64 k, i64 n, cudaStream_t s, int tile)
{
    if (m <= 0 || n <= 0) return MELA_OK;
    if (k <= 0) {
        MELA_CUDA_TRY(cudaMemset2DAsync(C, (size_t)ldc * 8, 0, (size_t)words_of(n) * 8, (size_t)m, s));
        return MELA_OK;
    }
    const i64 gx = (words_of(n) + M4_CTA_WORDS - 1) / M4_CTA_WORDS;
    const i64 gy = (m + M4_CTA_ROWS - 1) / M4_CTA_ROWS;
    if (mela_status st = check_grid_yz(gy, 1, "gemm_m4ri"); st != MELA_OK) return st;
    if (k > 0x7fffffffLL - 16) {
        set_error("gemm_m4ri: k beyond the TMA coordinate range");
        return MELA_ERR_UNSUPPORTED;
    }
    constexpr int smem = M4_SMEM_BYTES + 2 * M4_BTILE_WORDS * 8;
    CUtensorMap bmap;
    std::memset(&bmap, 0, sizeof bmap);
    // TMA reads B where its rows are 16-byte aligned
    const bool tma = (((uintptr_t)B & 15) == 0) && (ldb % 2 == 0) &&
                     make_u64_rows_map(&bmap, B, k, words_of(n), ldb, M4_CTA_WORDS, 16) == MELA_OK;
    u32 *err = device_error_word();
    const dim3 grid((unsigned)gx, (unsigned)gy);
    if (!tma) cudaGetLastError();
    auto launch = [&](auto kernel, int threads) -> mela_status {
        MELA_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        kernel<<<grid, threads, smem, s>>>(A, lda, B, ldb, C, ldc, m, k, n, bmap, err);
        return MELA_OK;
    };
    mela_status st;
    if (tile == 1)
        st = tma ? launch(gemm_m4ri_kernel<8, true>, 256) : launch(gemm_m4ri_kernel<8, false>, 256);
    else
        st = tma ? launch(gemm_m4ri_kernel<16, true>, 512) : launch(gemm_m4ri_kernel<16, false>, 512);
    if (st != MELA_OK) return st;
    MELA_LAUNCH_CHECK("gemm_m4ri_kernel");
    return MELA_OK;
}

}  // namespace mela
