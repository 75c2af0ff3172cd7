// gemm_plain.cu -- bit-packed GF(2) product on CUDA cores (AND + popcount parity).
//
// C(i,j) = parity( sum_k A(i,k) & B(k,j) ).  With the right operand held
// transposed (Bt, row j = column j of B), every 32 values of k cost one
// LOP3 per (i,j): acc ^= a & b, and the parity of acc's popcount at the end
// gives the bit.  This is the same product as the reference's XOR-row loop
// (src/mela_matmul_gf2.c:111-208) reorganised as an inner-product GEMM so
// that each thread keeps an 8x8 register tile of accumulators.
//
// CTA tile 128 (rows of A) x 128 (rows of Bt), 256 threads.  Thread (ty,tx)
// owns rows {4ty+a, 64+4ty+a} and columns {4tx+b, 64+4tx+b}, a,b in 0..3,
// so each shared-memory read of its operands is one conflict-free 16-byte
// vector.  K advances 512 bits per stage through double-buffered shared
// memory filled from registers prefetched one stage ahead.
#include "mela_common.cuh"
#include "mela_internal.h"

namespace mela {

namespace {

constexpr int TM = 128, TN = 128;
constexpr int KC = 16;          // u32 words of K per stage (512 bits)
constexpr int SP = TM + 4;      // padded shared row (u32)

struct Frag {
    u64 a[2][2];  // two u64 loads (2 x 16 bytes) of A per thread per stage
    u64 b[2][2];
};

__device__ __forceinline__ u64 ld_or_zero(const u64 *p, bool ok) { return ok ? __ldg(p) : 0ull; }

}  // namespace

__global__ void __launch_bounds__(256, 2)
gemm_plain_kernel(const u64 *__restrict__ A, i64 lda, const u64 *__restrict__ Bt, i64 ldb,
                  u64 *__restrict__ C, i64 ldc, i64 m, i64 n, i64 kw64)
{
    __shared__ __align__(16) u32 As[2][KC][SP];
    __shared__ __align__(16) u32 Bs[2][KC][SP];

    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const i64 i0 = (i64)blockIdx.y * TM;
    const i64 j0 = (i64)blockIdx.x * TN;

    // Loader mapping: tile has 128 rows x 8 u64 per stage = 1024 u64 per
    // operand; thread t loads u64 pairs (2 x 16 B) at flat indices t and t+256.
    // Pair p covers row p/4, u64 words 2*(p%4), 2*(p%4)+1 of the stage.
    auto load = [&](Frag &f, i64 kw0) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            int p = tid + h * 256;
            int r = p >> 2, q = p & 3;
            i64 w = kw0 + 2 * q;
            i64 ia = i0 + r, jb = j0 + r;
            bool ra = ia < m, rb = jb < n;
            f.a[h][0] = ld_or_zero(A + ia * lda + w, ra && w < kw64);
            f.a[h][1] = ld_or_zero(A + ia * lda + w + 1, ra && w + 1 < kw64);
            f.b[h][0] = ld_or_zero(Bt + jb * ldb + w, rb && w < kw64);
            f.b[h][1] = ld_or_zero(Bt + jb * ldb + w + 1, rb && w + 1 < kw64);
        }
    };
    auto store = [&](const Frag &f, int buf) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            int p = tid + h * 256;
            int r = p >> 2, q = p & 3;
            int k = 4 * q;  // u32 index within the stage
            As[buf][k + 0][r] = (u32)f.a[h][0];
            As[buf][k + 1][r] = (u32)(f.a[h][0] >> 32);
            As[buf][k + 2][r] = (u32)f.a[h][1];
            As[buf][k + 3][r] = (u32)(f.a[h][1] >> 32);
            Bs[buf][k + 0][r] = (u32)f.b[h][0];
            Bs[buf][k + 1][r] = (u32)(f.b[h][0] >> 32);
            Bs[buf][k + 2][r] = (u32)f.b[h][1];
            Bs[buf][k + 3][r] = (u32)(f.b[h][1] >> 32);
        }
    };

    u32 acc[8][8];
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < 8; ++b) acc[a][b] = 0;

    const i64 nstages = (kw64 + 7) / 8;
    Frag f;
    load(f, 0);
    store(f, 0);
    __syncthreads();

    for (i64 s = 0; s < nstages; ++s) {
        const int buf = (int)(s & 1);
        const bool more = s + 1 < nstages;
        if (more) load(f, (s + 1) * 8);
#pragma unroll
        for (int kk = 0; kk < KC; ++kk) {
            uint4 a0 = *reinterpret_cast<const uint4 *>(&As[buf][kk][4 * ty]);
            uint4 a1 = *reinterpret_cast<const uint4 *>(&As[buf][kk][64 + 4 * ty]);
            uint4 b0 = *reinterpret_cast<const uint4 *>(&Bs[buf][kk][4 * tx]);
            uint4 b1 = *reinterpret_cast<const uint4 *>(&Bs[buf][kk][64 + 4 * tx]);
            const u32 av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const u32 bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
            for (int a = 0; a < 8; ++a)
#pragma unroll
                for (int b = 0; b < 8; ++b) acc[a][b] ^= av[a] & bv[b];
        }
        if (more) store(f, buf ^ 1);
        __syncthreads();
    }

    // Epilogue: bit (row, col) = parity(acc).  Row 4ty+a (a<4) or
    // 64+4ty+(a-4) holds, in this thread, nibble tx of word 0 (b<4) and
    // nibble tx of word 1 (b>=4); OR-reduce the 16 nibbles over the 16
    // lanes sharing ty.
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        u32 lo = 0, hi = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            lo |= (u32)(__popc(acc[a][b]) & 1) << b;
            hi |= (u32)(__popc(acc[a][b + 4]) & 1) << b;
        }
        u64 w0 = (u64)lo << (4 * tx);
        u64 w1 = (u64)hi << (4 * tx);
#pragma unroll
        for (int o = 1; o < 16; o <<= 1) {
            w0 |= __shfl_xor_sync(0xffffffffu, w0, o);
            w1 |= __shfl_xor_sync(0xffffffffu, w1, o);
        }
        const i64 row = i0 + (a < 4 ? 4 * ty + a : 64 + 4 * ty + (a - 4));
        if (row < m) {
            const i64 wj = j0 >> 6;
            const i64 nw = words_of(n);
            if (tx == 0 && wj < nw) C[row * ldc + wj] = w0;
            if (tx == 1 && wj + 1 < nw) C[row * ldc + wj + 1] = w1;
        }
    }
}

mela_status launch_gemm_plain(const u64 *A, i64 lda, const u64 *Bt, i64 ldbt, u64 *C, i64 ldc,
                              i64 m, i64 k, i64 n, cudaStream_t s)
{
    if (m <= 0 || n <= 0) return MELA_OK;
    if (k <= 0) {
        MELA_CUDA_TRY(cudaMemset2DAsync(C, (size_t)ldc * 8, 0, (size_t)words_of(n) * 8, (size_t)m, s));
        return MELA_OK;
    }
    dim3 grid((unsigned)((n + TN - 1) / TN), (unsigned)((m + TM - 1) / TM));
    if (grid.y > 65535u) {
        set_error("gemm_plain: m too large for one launch");
        return MELA_ERR_UNSUPPORTED;
    }
    gemm_plain_kernel<<<grid, 256, 0, s>>>(A, lda, Bt, ldbt, C, ldc, m, n, words_of(k));
    MELA_LAUNCH_CHECK("gemm_plain_kernel");
    return MELA_OK;
}

}  // namespace mela
