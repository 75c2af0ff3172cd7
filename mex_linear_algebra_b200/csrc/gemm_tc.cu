// gemm_tc.cu -- GF(2) product on the sm_100a tensor cores (tcgen05, kind::i8).
//
// Both operands are 0/1 bytes (expanded from the packed bits by
// expand_u8_kernel), K-major: A8 is m x k, Bt8 is n x k (B transposed).  The
// tensor cores accumulate the integer dot products in 32-bit TMEM cells;
// bit (i,j) of the GF(2) product is the low bit of the sum.  The sum is at
// most k < 2^31, and the low bit of a 32-bit two's-complement sum is exact
// even past that, so the result is bit-exact for every k.
//
// Kernel structure (one 128 x 256 output tile per CTA, 192 threads):
//   warp 0  lane 0 : TMA producer, 4-stage ring of (A 128x128 B, B 256x128 B)
//   warp 1         : allocates 256 TMEM columns; lane 0 issues 4 UMMAs of
//                    K=32 per stage and commits each stage back to its
//                    producer barrier
//   warps 2..5     : epilogue; each reads its 32 TMEM lanes (= 32 output
//                    rows) x 256 columns, keeps the parity bit and writes 4
//                    packed words per row.
// Tiles are rasterised in bands of 16 tile-rows so that the CTAs resident
// at one time share A and B tiles in L2.
//
// FP4 form (F4 = true): the operands are packed E2M1 values (0x2 = 1.0,
// 0x0 = 0; two per byte), the instruction is tcgen05 kind::mxf4 with one
// UE8M0 scale factor per 32 values of K, at twice the INT8 rate.  Every scale
// factor is 1.0, so the scale-factor columns of TMEM are one constant block
// (bytes 0x7F) written once per CTA and addressed by every instruction.  The
// f32 accumulator holds the integer dot product exactly; K < 2^23 is
// required so that adding 2^23 puts the integer in the low mantissa bits,
// whose bit 0 is the parity (one float add per value instead of a
// float-to-int conversion).
#include <cstdlib>

#include "mela_common.cuh"
#include "mela_internal.h"
#include "tc_ptx.cuh"

namespace mela {

namespace {

constexpr int BM = 128, BN = 256, BK = 128;  // BK in bytes (= K elements)
constexpr int STAGES = 4;
constexpr int A_BYTES = BM * BK;
constexpr int B_BYTES = BN * BK;
constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;
constexpr u32 SF_COL = 256;   // first TMEM column of the 32 constant scale-factor columns (FP4 form)
constexpr int GROUP_M = 16;

struct Ctl {
    u64 full[STAGES];
    u64 empty[STAGES];
    u64 acc;
    u64 drain;
    u32 tmem;
    int abort;
};

}  // namespace

template <bool F4>
__global__ void __launch_bounds__(192, 1)
gemm_tc_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
               u64 *__restrict__ C, i64 ldc, i64 m, i64 n, int tiles_m, int tiles_n, int kstages,
               u32 *err)
{
    constexpr u32 TMEM_COLS = F4 ? 512 : 256;
    extern __shared__ unsigned char smem_raw[];
    unsigned char *smem =
        reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    Ctl *ctl = reinterpret_cast<Ctl *>(smem + STAGES * STAGE_BYTES);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    // grouped rasterisation
    const int t = blockIdx.x;
    const int per_group = GROUP_M * tiles_n;
    const int group = t / per_group;
    const int first_m = group * GROUP_M;
    const int gsize = (tiles_m - first_m) < GROUP_M ? (tiles_m - first_m) : GROUP_M;
    const int tm = first_m + (t % per_group) % gsize;
    const int tn = (t % per_group) / gsize;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            ptx::mbar_init(&ctl->full[s], 1);
            ptx::mbar_init(&ctl->empty[s], 1);
        }
        ptx::mbar_init(&ctl->acc, 1);
        ptx::mbar_init(&ctl->drain, 1);
        ctl->abort = 0;
        ptx::fence_barrier_init();
    }
    if (warp == 0 && lane == 0) {
        ptx::prefetch_tmap(&tmA);
        ptx::prefetch_tmap(&tmB);
    }
    if (warp == 1) {
        ptx::tmem_alloc(&ctl->tmem, TMEM_COLS);
        ptx::tmem_relinquish();
    }
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    const u32 tmem = ctl->tmem;
    volatile int *abort_flag = &ctl->abort;
    if constexpr (F4) {
        // constant scale factors: every byte of columns SF_COL.. = 0x7F (2^0)
        if (warp >= 2) {
            const u32 lane_base = (u32)((warp & 3) * 32) << 16;
            ptx::tmem_st_32x32b_x16(tmem + lane_base + SF_COL, 0x7F7F7F7Fu);
            ptx::tmem_st_32x32b_x16(tmem + lane_base + SF_COL + 16, 0x7F7F7F7Fu);
            ptx::tmem_st_wait();
        }
        ptx::tc_fence_before();
        __syncthreads();
        ptx::tc_fence_after();
    }

    if (warp == 0) {
        if (lane == 0) {
            int last_round[STAGES];
#pragma unroll
            for (int s = 0; s < STAGES; ++s) last_round[s] = -1;
            for (int ks = 0; ks < kstages; ++ks) {
                const int s = ks % STAGES, round = ks / STAGES;
                if (round > 0 && !ptx::mbar_wait(&ctl->empty[s], (round - 1) & 1, err)) {
                    *abort_flag = 1;
                    break;
                }
                if (*abort_flag) break;
                unsigned char *sa = smem + s * STAGE_BYTES;
                ptx::mbar_arrive_expect_tx(&ctl->full[s], STAGE_BYTES);
                ptx::tma_load_2d(sa, &tmA, &ctl->full[s], ks * BK, tm * BM);
                ptx::tma_load_2d(sa + A_BYTES, &tmB, &ctl->full[s], ks * BK, tn * BN);
                last_round[s] = round;
            }
            if (*abort_flag) {
                // let every issued copy land before the CTA's shared memory goes away
                for (int s = 0; s < STAGES; ++s)
                    if (last_round[s] >= 0) ptx::mbar_wait(&ctl->full[s], last_round[s] & 1, nullptr);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            constexpr u32 idesc = F4 ? ptx::idesc_mxf4(BM, BN) : ptx::idesc_i8(BM, BN);
            bool ok = true;
            for (int ks = 0; ks < kstages; ++ks) {
                const int s = ks % STAGES, round = ks / STAGES;
                if (!ptx::mbar_wait(&ctl->full[s], round & 1, err) || *abort_flag) {
                    *abort_flag = 1;
                    ok = false;
                    break;
                }
                ptx::tc_fence_after();
                const u32 a0 = ptx::smem_u32(smem + s * STAGE_BYTES);
                const u32 b0 = a0 + A_BYTES;
#pragma unroll
                for (int kk = 0; kk < BK / 32; ++kk) {
                    // 32 bytes of K per instruction: 32 int8 values or 64 packed e2m1 values
                    if constexpr (F4)
                        ptx::umma_mxf4(tmem, ptx::desc_k_sw128(a0 + kk * 32), ptx::desc_k_sw128(b0 + kk * 32),
                                       idesc, tmem + SF_COL, tmem + SF_COL + 8, (ks | kk) != 0);
                    else
                        ptx::umma_i8(tmem, ptx::desc_k_sw128(a0 + kk * 32), ptx::desc_k_sw128(b0 + kk * 32),
                                     idesc, (ks | kk) != 0);
                }
                ptx::umma_commit(&ctl->empty[s]);
            }
            if (ok) {
                ptx::umma_commit(&ctl->acc);
            } else {
                // drain UMMAs still reading shared memory, then release the epilogue
                ptx::umma_commit(&ctl->drain);
                ptx::mbar_wait(&ctl->drain, 0, nullptr);
                ptx::mbar_arrive(&ctl->acc);
            }
        }
        __syncwarp();
    } else {
        const bool ok = ptx::mbar_wait(&ctl->acc, 0, err);
        ptx::tc_fence_after();
        if (ok && !*abort_flag) {
            const int ew = warp & 3;  // TMEM lane quarter this warp may access
            const i64 row = (i64)tm * BM + ew * 32 + lane;
            u32 bits[BN / 32];
#pragma unroll
            for (int c = 0; c < BN / 32; ++c) {
                u32 r[32];
                ptx::tmem_ld_32x32b_x32(tmem + ((u32)(ew * 32) << 16) + (u32)(c * 32), r);
                ptx::tmem_ld_wait();
                u32 b = 0;
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const u32 v = F4 ? __float_as_uint(__uint_as_float(r[j]) + 8388608.0f) : r[j];
                    b |= (v & 1u) << j;
                }
                bits[c] = b;
            }
            const i64 nw = words_of(n);
            if (row < m) {
#pragma unroll
                for (int q = 0; q < BN / 64; ++q) {
                    const i64 w = (i64)tn * (BN / 64) + q;
                    if (w < nw) C[row * ldc + w] = (u64)bits[2 * q] | ((u64)bits[2 * q + 1] << 32);
                }
            }
        }
    }

    ptx::tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        ptx::tc_fence_after();
        ptx::tmem_dealloc(tmem, TMEM_COLS);
    }
}

// ---------------------------------------------------------------- CTA pairs
// The same product with 256 x 256 output tiles computed by a cluster of two
// CTAs (tcgen05 cta_group::2).  CTA r of the pair loads rows r*128..+127 of
// the tile's A rows and of its B rows (B transposed) into its own shared
// memory; the TMA completions of both CTAs are counted on the even CTA's
// stage barrier, and the even CTA's MMA thread issues M = 256 instructions
// that read both CTAs' halves and accumulate, in each CTA's TMEM, that CTA's
// 128 rows x 256 columns.  Each SM thereby fills half as many B bytes into
// shared memory per instruction as with one CTA per tile.  The MMA commits
// arrive on the barrier of the same offset in both CTAs, so each CTA's
// producer learns when a stage is free and each CTA's epilogue when its
// accumulator is ready.  No TMA load uses cluster multicast.
namespace {
constexpr int P_STAGES = 7;
constexpr int P_A_BYTES = 128 * BK;                    // this CTA's 128 rows of A
constexpr int P_B_BYTES = 128 * BK;                    // this CTA's 128 rows of B
constexpr int P_STAGE_BYTES = P_A_BYTES + P_B_BYTES;
constexpr int P_SMEM_BYTES = P_STAGES * P_STAGE_BYTES + 1024 + 256;

struct PairCtl {
    u64 full[P_STAGES];   // even CTA: both CTAs' bytes of a stage have landed
    u64 empty[P_STAGES];  // both CTAs: the pair's MMAs have read a stage
    u64 acc_full;         // both CTAs: the accumulator holds a finished tile
    u64 acc_empty;        // even CTA: both CTAs' epilogues have read the accumulator
    u64 drain;
    u32 tmem;
    int abort;
};
constexpr int P_EPI_WARPS = 4;
}  // namespace

// Persistent: cluster c computes tiles c, c + clusters, ... (grouped
// rasterisation over 256 x 256 tiles).  The stage ring runs on across tiles,
// so the producer fills the next tile's stages while the current tile's last
// MMAs and its epilogue run; the MMA thread starts a tile once both CTAs'
// epilogues have read the previous one out of TMEM.
template <bool F4>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(192, 1)
gemm_tc_pair_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                    u64 *__restrict__ C, i64 ldc, i64 m, i64 n, int tiles_m, int tiles_n, int kstages, u32 *err)
{
    constexpr u32 TMEM_COLS = F4 ? 512 : 256;
    extern __shared__ unsigned char smem_raw[];
    unsigned char *smem =
        reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    PairCtl *ctl = reinterpret_cast<PairCtl *>(smem + P_STAGES * P_STAGE_BYTES);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const u32 rank = ptx::cluster_ctarank();
    const bool leader = rank == 0;
    const int cid = blockIdx.x >> 1, clusters = gridDim.x >> 1;
    const int ntiles = tiles_m * tiles_n;
    auto coords = [&](int t, int &tm, int &tn) {
        const int per_group = GROUP_M * tiles_n;
        const int group = t / per_group;
        const int first_m = group * GROUP_M;
        const int gsize = (tiles_m - first_m) < GROUP_M ? (tiles_m - first_m) : GROUP_M;
        tm = first_m + (t % per_group) % gsize;
        tn = (t % per_group) / gsize;
    };

    if (threadIdx.x == 0) {
        for (int s = 0; s < P_STAGES; ++s) {
            ptx::mbar_init(&ctl->full[s], 1);
            ptx::mbar_init(&ctl->empty[s], 1);
        }
        ptx::mbar_init(&ctl->acc_full, 1);
        ptx::mbar_init(&ctl->acc_empty, 2 * P_EPI_WARPS);
        ptx::mbar_init(&ctl->drain, 1);
        ctl->abort = 0;
        ptx::fence_barrier_init();
    }
    if (warp == 0 && lane == 0) {
        ptx::prefetch_tmap(&tmA);
        ptx::prefetch_tmap(&tmB);
    }
    if (warp == 1) {
        ptx::tmem_alloc_pair(&ctl->tmem, TMEM_COLS);
        ptx::tmem_relinquish_pair();
    }
    ptx::tc_fence_before();
    ptx::cluster_sync();  // both CTAs' barriers and TMEM exist before any copy or MMA
    ptx::tc_fence_after();
    const u32 tmem = ctl->tmem;
    volatile int *abort_flag = &ctl->abort;
    if constexpr (F4) {
        if (warp >= 2) {
            const u32 lane_base = (u32)((warp & 3) * 32) << 16;
            ptx::tmem_st_32x32b_x16(tmem + lane_base + SF_COL, 0x7F7F7F7Fu);
            ptx::tmem_st_32x32b_x16(tmem + lane_base + SF_COL + 16, 0x7F7F7F7Fu);
            ptx::tmem_st_wait();
        }
        ptx::tc_fence_before();
        ptx::cluster_sync();  // the scale factors of both CTAs are in place
        ptx::tc_fence_after();
    }

    if (warp == 0) {
        if (lane == 0) {
            const u32 full0 = ptx::mapa_shared(ptx::smem_u32(&ctl->full[0]), 0);
            int g = 0;  // stage counter over all tiles of this cluster
            bool ok = true;
            for (int t = cid; t < ntiles && ok; t += clusters) {
                int tm, tn;
                coords(t, tm, tn);
                for (int ks = 0; ks < kstages; ++ks, ++g) {
                    const int s = g % P_STAGES, round = g / P_STAGES;
                    if ((round > 0 && !ptx::mbar_wait(&ctl->empty[s], (round - 1) & 1, err)) || *abort_flag) {
                        *abort_flag = 1;
                        ok = false;
                        break;
                    }
                    unsigned char *sa = smem + s * P_STAGE_BYTES;
                    if (leader) ptx::mbar_arrive_expect_tx(&ctl->full[s], 2 * P_STAGE_BYTES);
                    const u32 bar = full0 + (u32)(s * sizeof(u64));
                    ptx::tma_load_2d_pair(sa, &tmA, bar, ks * BK, tm * 256 + (int)rank * 128);
                    ptx::tma_load_2d_pair(sa + P_A_BYTES, &tmB, bar, ks * BK, tn * 256 + (int)rank * 128);
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0 && leader) {
            constexpr u32 idesc = F4 ? ptx::idesc_mxf4(256, BN) : ptx::idesc_i8(256, BN);
            bool ok = true;
            int g = 0, i = 0;
            for (int t = cid; t < ntiles && ok; t += clusters, ++i) {
                // the previous tile has left TMEM (both CTAs)
                if (i > 0 && (!ptx::mbar_wait_cluster(&ctl->acc_empty, (i - 1) & 1, err) || *abort_flag)) {
                    ok = false;
                    break;
                }
                ptx::tc_fence_after();
                for (int ks = 0; ks < kstages; ++ks, ++g) {
                    const int s = g % P_STAGES, round = g / P_STAGES;
                    if (!ptx::mbar_wait(&ctl->full[s], round & 1, err) || *abort_flag) {
                        ok = false;
                        break;
                    }
                    ptx::tc_fence_after();
                    const u32 a0 = ptx::smem_u32(smem + s * P_STAGE_BYTES);
                    const u32 b0 = a0 + P_A_BYTES;
#pragma unroll
                    for (int kk = 0; kk < BK / 32; ++kk) {
                        if constexpr (F4)
                            ptx::umma_mxf4_pair(tmem, ptx::desc_k_sw128(a0 + kk * 32),
                                                ptx::desc_k_sw128(b0 + kk * 32), idesc, tmem + SF_COL,
                                                tmem + SF_COL + 8, (ks | kk) != 0);
                        else
                            ptx::umma_i8_pair(tmem, ptx::desc_k_sw128(a0 + kk * 32), ptx::desc_k_sw128(b0 + kk * 32),
                                              idesc, (ks | kk) != 0);
                    }
                    ptx::umma_commit_pair(&ctl->empty[s], 0x3);
                }
                if (ok) ptx::umma_commit_pair(&ctl->acc_full, 0x3);
            }
            if (!ok) {
                *abort_flag = 1;
                // drain the MMAs still reading either CTA's shared memory
                ptx::umma_commit_pair(&ctl->drain, 0x1);
                ptx::mbar_wait(&ctl->drain, 0, nullptr);
            }
        }
        __syncwarp();
    } else {
        const int ew = warp & 3;  // TMEM lane quarter this warp may access
        const u32 acc_empty0 = ptx::mapa_shared(ptx::smem_u32(&ctl->acc_empty), 0);
        const i64 nw = words_of(n);
        int i = 0;
        for (int t = cid; t < ntiles; t += clusters, ++i) {
            const bool ok = ptx::mbar_wait(&ctl->acc_full, i & 1, err);
            ptx::tc_fence_after();
            if (!ok || *abort_flag) {
                *abort_flag = 1;
                break;
            }
            int tm, tn;
            coords(t, tm, tn);
            const i64 row = (i64)tm * 256 + (i64)rank * 128 + ew * 32 + lane;
            u32 bits[BN / 32];
#pragma unroll
            for (int c = 0; c < BN / 32; ++c) {
                u32 r[32];
                ptx::tmem_ld_32x32b_x32(tmem + ((u32)(ew * 32) << 16) + (u32)(c * 32), r);
                ptx::tmem_ld_wait();
                u32 b = 0;
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const u32 v = F4 ? __float_as_uint(__uint_as_float(r[j]) + 8388608.0f) : r[j];
                    b |= (v & 1u) << j;
                }
                bits[c] = b;
            }
            // this warp's TMEM reads are done: the next tile may overwrite them
            ptx::tc_fence_before();
            __syncwarp();
            if (lane == 0) ptx::mbar_arrive_cluster(acc_empty0);
            if (row < m) {
#pragma unroll
                for (int q = 0; q < BN / 64; ++q) {
                    const i64 w = (i64)tn * (BN / 64) + q;
                    if (w < nw) C[row * ldc + w] = (u64)bits[2 * q] | ((u64)bits[2 * q + 1] << 32);
                }
            }
        }
    }

    ptx::tc_fence_before();
    __syncthreads();
    ptx::cluster_sync();  // neither CTA leaves while the pair's MMAs may still read its shared memory
    if (warp == 1) {
        ptx::tc_fence_after();
        ptx::tmem_dealloc_pair(tmem, TMEM_COLS);
    }
}

// ---------------------------------------------------------------- host side
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    }
    return fn;
}

// K-major byte matrix rows x kp, box (128 bytes, box_rows rows), 128-byte swizzle.
static mela_status make_map(CUtensorMap *map, const unsigned char *base, i64 rows, i64 kp,
                            int box_rows)
{
    EncodeTiledFn fn = encode_fn();
    if (!fn) {
        set_error("cuTensorMapEncodeTiled unavailable");
        return MELA_ERR_CUDA;
    }
    cuuint64_t dims[2] = {(cuuint64_t)kp, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)kp};
    cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, (void *)base, dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
        return MELA_ERR_CUDA;
    }
    return MELA_OK;
}

mela_status make_u8_kmajor_map(CUtensorMap *map, const unsigned char *base, i64 rows, i64 kp, int box_rows)
{
    return make_map(map, base, rows, kp, box_rows);
}

mela_status make_u64_rows_map(CUtensorMap *map, const u64 *base, i64 rows, i64 words, i64 ld, int box_words,
                              int box_rows)
{
    EncodeTiledFn fn = encode_fn();
    if (!fn) {
        set_error("cuTensorMapEncodeTiled unavailable");
        return MELA_ERR_CUDA;
    }
    cuuint64_t dims[2] = {(cuuint64_t)words, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ld * 8};
    cuuint32_t box[2] = {(cuuint32_t)box_words, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT64, 2, (void *)base, dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled (packed rows) failed (%d)", (int)r);
        return MELA_ERR_CUDA;
    }
    return MELA_OK;
}

// CTA pairs are used whenever the padded row count allows (mp % 256 == 0),
// unless the tile choice asks for single CTAs (tile 1) or, for the default
// choice, MELA_TC_PAIR=0 is set in the environment.
static bool use_pairs(i64 mp, int tile)
{
    if (mp % 256 || tile == 1) return false;
    if (tile == 2) return true;
    const char *e = getenv("MELA_TC_PAIR");
    return !(e && e[0] == '0');
}

mela_status launch_gemm_tc(const unsigned char *A8, const unsigned char *Bt8, i64 mp, i64 np,
                           i64 kp, u64 *C, i64 ldc, i64 m, i64 n, cudaStream_t s, bool fp4, int tile)
{
    if (m <= 0 || n <= 0) return MELA_OK;
    if (mp % BM || np % BN || kp % BK || kp <= 0) {
        set_error("gemm_tc: padded shape %lld x %lld x %lld not tile-aligned", mp, np, kp);
        return MELA_ERR_INVALID;
    }
    if (((uintptr_t)A8 | (uintptr_t)Bt8) & 15) {
        set_error("gemm_tc: operands must be 16-byte aligned");
        return MELA_ERR_INVALID;
    }
    const i64 tiles_m = mp / BM, tiles_n = np / BN, kst = kp / BK;
    if (tiles_m * tiles_n > 0x7fffffffLL || kst > 0x7fffffffLL || kp > (1LL << 31)) {
        set_error("gemm_tc: problem too large for one launch");
        return MELA_ERR_UNSUPPORTED;
    }
    if (use_pairs(mp, tile)) {
        CUtensorMap ma, mb;
        mela_status st = make_map(&ma, A8, mp, kp, 128);
        if (st != MELA_OK) return st;
        st = make_map(&mb, Bt8, np, kp, 128);
        if (st != MELA_OK) return st;
        const i64 ntiles = (mp / 256) * tiles_n, clusters_max = sm_count() / 2;
        const unsigned grid = (unsigned)(2 * (ntiles < clusters_max ? ntiles : clusters_max));
        if (fp4) {
            MELA_CUDA_TRY(cudaFuncSetAttribute(gemm_tc_pair_kernel<true>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, P_SMEM_BYTES));
            gemm_tc_pair_kernel<true><<<grid, 192, P_SMEM_BYTES, s>>>(ma, mb, C, ldc, m, n, (int)(mp / 256),
                                                                       (int)tiles_n, (int)kst, device_error_word());
        } else {
            MELA_CUDA_TRY(cudaFuncSetAttribute(gemm_tc_pair_kernel<false>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, P_SMEM_BYTES));
            gemm_tc_pair_kernel<false><<<grid, 192, P_SMEM_BYTES, s>>>(ma, mb, C, ldc, m, n, (int)(mp / 256),
                                                                        (int)tiles_n, (int)kst, device_error_word());
        }
        MELA_LAUNCH_CHECK("gemm_tc_pair_kernel");
        return MELA_OK;
    }
    CUtensorMap ma, mb;
    mela_status st = make_map(&ma, A8, mp, kp, BM);
    if (st != MELA_OK) return st;
    st = make_map(&mb, Bt8, np, kp, BN);
    if (st != MELA_OK) return st;
    if (fp4) {
        MELA_CUDA_TRY(cudaFuncSetAttribute(gemm_tc_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           SMEM_BYTES));
        gemm_tc_kernel<true><<<(unsigned)(tiles_m * tiles_n), 192, SMEM_BYTES, s>>>(
            ma, mb, C, ldc, m, n, (int)tiles_m, (int)tiles_n, (int)kst, device_error_word());
    } else {
        MELA_CUDA_TRY(cudaFuncSetAttribute(gemm_tc_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           SMEM_BYTES));
        gemm_tc_kernel<false><<<(unsigned)(tiles_m * tiles_n), 192, SMEM_BYTES, s>>>(
            ma, mb, C, ldc, m, n, (int)tiles_m, (int)tiles_n, (int)kst, device_error_word());
    }
    MELA_LAUNCH_CHECK("gemm_tc_kernel");
    return MELA_OK;
}

}  // namespace mela
