// pack.cu -- data-format kernels on the path into and out of the GF(2) kernels.
//
//  * rand_dense   seeded Bernoulli(1/2) packed matrices (counter-based
//                 splitmix64, identical bits to the CPU generator)
//  * pack         MATLAB column-major logical / double -> packed rows
//                 (reference: pack_rows_logical / pack_rows_double,
//                 src/mela_matmul_gf2.c:42-69; inline packs in
//                 src/mela_rank_gf2.c:154-176, src/mela_null_gf2.c:169-187)
//  * unpack       packed rows -> column-major logical bytes
//                 (reference: src/mela_matmul_gf2.c:193-205)
//  * transpose    64x64 bit-block transpose with warp ballots
//  * expand_u8    packed bits -> 0/1 bytes (operands of the tensor-core GEMM)
//
// All of these are HBM-bound byte/word moves: each thread reads and writes
// whole words or bytes with warp-contiguous addresses; no GEMM reshaping.
#include "mela_common.cuh"
#include "mela_internal.h"

namespace mela {

// ---------------------------------------------------------------- generator
__host__ __device__ __forceinline__ u64 mix64(u64 z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

u64 stream_key(u64 seed, u64 stream)
{
    return mix64(seed * 0x9E3779B97F4A7C15ULL + 0x632BE59BD9B4E019ULL) ^
           mix64(stream + 0xD1B54A32D192ED03ULL);
}

__global__ void rand_dense_kernel(u64 key, i64 m, i64 n, i64 wc, u64 *out, i64 ld)
{
    const u64 tail = (n & 63) ? ((1ULL << (n & 63)) - 1) : ~0ULL;
    i64 total = m * ld;
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < total;
         t += (i64)gridDim.x * blockDim.x) {
        i64 i = t / ld, w = t - i * ld;
        u64 v = 0;
        if (w < wc) {
            v = mix64(key + (u64)(i * wc + w + 1) * 0x9E3779B97F4A7C15ULL);
            if (w == wc - 1) v &= tail;
        }
        out[t] = v;
    }
}

// Bernoulli(density) bits: entry e = i*n + j takes 16-bit slice e%4 of word
// e/4 of the stream and is 1 when the slice is below `thresh` (density*65536).
__global__ void rand_bernoulli_kernel(u64 key, i64 m, i64 n, unsigned thresh, u64 *out, i64 ld)
{
    const i64 wc = words_of(n);
    const i64 total = m * ld;
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < total; t += (i64)gridDim.x * blockDim.x) {
        const i64 i = t / ld, w = t - i * ld;
        u64 v = 0;
        if (w < wc) {
            const int cols = (n - 64 * w) < 64 ? (int)(n - 64 * w) : 64;
            for (int b = 0; b < cols; ++b) {
                const i64 e = i * n + 64 * w + b;
                const u64 word = mix64(key + (u64)(e / 4 + 1) * 0x9E3779B97F4A7C15ULL);
                const unsigned sl = (unsigned)(word >> (16 * (e & 3))) & 0xFFFFu;
                if (sl < thresh) v |= 1ull << b;
            }
        }
        out[t] = v;
    }
}

// ---------------------------------------------------------------- pack
// Parity of a double as the reference reads it, ((int)x) & 1, with the
// x86-64 result for NaN and out-of-range values (INT_MIN, even) spelled out.
__device__ __forceinline__ u32 parity_of(double x)
{
    if (!(x >= -2147483648.0 && x < 2147483648.0)) return 0;
    return (u32)__double2int_rz(x) & 1u;
}
__device__ __forceinline__ u32 parity_of(unsigned char x) { return x != 0; }

// One block: 32 rows x 8 output words (512 columns).  Warp w builds word
// column w: lane l owns row row0+l and walks the 64 columns of its word,
// so each load instruction reads 32 consecutive rows of one column.
template <typename T>
__global__ void __launch_bounds__(256) pack_kernel(const T *__restrict__ in, i64 m, i64 n,
                                                   u64 *__restrict__ out, i64 ld, i64 out_words)
{
    __shared__ u64 tile[32][9];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const i64 row0 = (i64)blockIdx.x * 32;
    const i64 w = (i64)blockIdx.y * 8 + warp;
    const i64 row = row0 + lane;
    u64 word = 0;
    if (row < m && w * 64 < n) {
        const i64 c0 = w * 64;
        const int cols = (int)((n - c0) < 64 ? (n - c0) : 64);
        const T *p = in + row + c0 * m;
        for (int j = 0; j < cols; ++j) word |= (u64)parity_of(p[(i64)j * m]) << j;
    }
    tile[lane][warp] = word;
    __syncthreads();
    const int r = threadIdx.x >> 3, q = threadIdx.x & 7;
    const i64 orow = row0 + r, ow = (i64)blockIdx.y * 8 + q;
    if (orow < m && ow < out_words) out[orow * ld + ow] = tile[r][q];
}

// ---------------------------------------------------------------- unpack
// One warp: 32 rows x 64 columns; each store instruction writes 32
// consecutive rows of one column (column-major output).
__global__ void __launch_bounds__(256) unpack_kernel(const u64 *__restrict__ in, i64 ld, i64 m,
                                                     i64 n, unsigned char *__restrict__ out)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const i64 row = (i64)blockIdx.x * 32 + lane;
    const i64 w = (i64)blockIdx.y * 8 + warp;
    if (w * 64 >= n) return;
    const i64 c0 = w * 64;
    const int cols = (int)((n - c0) < 64 ? (n - c0) : 64);
    if (row >= m) return;
    u64 word = in[row * ld + w];
    unsigned char *p = out + row + c0 * m;
    for (int j = 0; j < cols; ++j) p[(i64)j * m] = (unsigned char)((word >> j) & 1);
}

// ---------------------------------------------------------------- transpose
// Block: 256 input rows x 64 input columns.  Warp w loads rows
// 32w..32w+31 (one word each); two 32x32 warp transposes give, per input
// column b, the 32 bits of rows 32w..32w+31.  Output row (column b) receives
// 4 words.
__global__ void __launch_bounds__(256) transpose_kernel(const u64 *__restrict__ in, i64 ld_in,
                                                        i64 rows, i64 cols,
                                                        u64 *__restrict__ out, i64 ld_out)
{
    __shared__ u32 part[8][65];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const i64 wcol = blockIdx.x;           // input word column
    const i64 r0 = (i64)blockIdx.y * 256;  // input row group
    const i64 row = r0 + warp * 32 + lane;
    u64 x = (row < rows) ? in[row * ld_in + wcol] : 0ull;
    const u32 keep0 = transpose32_warp((u32)x), keep1 = transpose32_warp((u32)(x >> 32));
    part[warp][lane] = keep0;
    part[warp][lane + 32] = keep1;
    __syncthreads();
    const int b = threadIdx.x >> 2, q = threadIdx.x & 3;
    const i64 ocol_row = wcol * 64 + b;  // output row index
    const i64 ow = (i64)blockIdx.y * 4 + q;
    const i64 owc = words_of(rows);
    if (ocol_row < cols && ow < owc)
        out[ocol_row * ld_out + ow] = (u64)part[2 * q][b] | ((u64)part[2 * q + 1][b] << 32);
}

// ---------------------------------------------------------------- expand to bytes
// out[r][k] = bit k of packed row r, for r < rows_pad, k < kpad (multiple of
// 64); zero outside rows x kbits.  One thread per 64-bit word -> 64 bytes.
__device__ __forceinline__ u32 spread4(u32 nib) { return (nib * 0x00204081u) & 0x01010101u; }

__global__ void __launch_bounds__(256) expand_u8_kernel(const u64 *__restrict__ in, i64 ld,
                                                        i64 rows, i64 kbits, i64 rows_pad,
                                                        i64 kpad, unsigned char *__restrict__ out)
{
    const i64 wpr = kpad >> 6;  // words per padded row
    const i64 total = rows_pad * wpr;
    const i64 wc = words_of(kbits);
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < total;
         t += (i64)gridDim.x * blockDim.x) {
        const i64 r = t / wpr, w = t - r * wpr;
        u64 v = (r < rows && w < wc) ? in[r * ld + w] : 0ull;
        uint4 *dst = reinterpret_cast<uint4 *>(out + r * kpad + w * 64);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            u32 h = (u32)(v >> (16 * q));
            uint4 o;
            o.x = spread4(h & 15);
            o.y = spread4((h >> 4) & 15);
            o.z = spread4((h >> 8) & 15);
            o.w = spread4((h >> 12) & 15);
            dst[q] = o;
        }
    }
}

// out (rows_pad x kpad_bytes, two e2m1 values per byte): value k of row r is
// 1.0 (0x2) when bit k of packed row r is set, else 0; element 2j in the low
// nibble of byte j.  One thread per 64-bit word -> 32 bytes.
__device__ __forceinline__ u32 spread_even4(u32 v)  // bits 0,2,4,6 -> bit 0 of bytes 0..3
{
    return (v & 1u) | ((v & 4u) << 6) | ((v & 16u) << 12) | ((v & 64u) << 18);
}

__global__ void __launch_bounds__(256) expand_f4_kernel(const u64 *__restrict__ in, i64 ld, i64 rows,
                                                        i64 kbits, i64 rows_pad, i64 kpad_bytes,
                                                        unsigned char *__restrict__ out)
{
    const i64 wpr = kpad_bytes >> 5;  // 64-bit source words per padded row
    const i64 total = rows_pad * wpr;
    const i64 wc = words_of(kbits);
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < total;
         t += (i64)gridDim.x * blockDim.x) {
        const i64 r = t / wpr, w = t - r * wpr;
        const u64 v = (r < rows && w < wc) ? in[r * ld + w] : 0ull;
        u32 o[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const u32 x = (u32)(v >> (8 * q)) & 0xFFu;
            o[q] = (spread_even4(x & 0x55u) << 1) | (spread_even4((x >> 1) & 0x55u) << 5);
        }
        uint4 *dst = reinterpret_cast<uint4 *>(out + r * kpad_bytes + w * 32);
        dst[0] = make_uint4(o[0], o[1], o[2], o[3]);
        dst[1] = make_uint4(o[4], o[5], o[6], o[7]);
    }
}

// Transposing expansion: out row j (j < cols_pad) holds column j of the packed
// kbits x cols matrix `in` as K-major tensor-core values -- 0/1 bytes (F4 =
// false, kpad bytes per row) or e2m1 pairs (F4 = true, kpad bytes per row =
// two values each) -- zero past kbits and past cols.  It replaces a bit
// transpose followed by an expansion.  Block: 256 k x 256 columns.  Each
// warp reads 32 rows of 256 bits (a lane per row) and turns them into
// 32-bit column slices by five rounds of shuffle butterflies; the output rows
// are written in 16-byte pieces, contiguous along k.
template <bool F4>
__global__ void __launch_bounds__(256) expand_t_kernel(const u64 *__restrict__ in, i64 ld, i64 kbits, i64 cols,
                                                       i64 kpad, unsigned char *__restrict__ out)
{
    __shared__ u32 U[256][9];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const i64 j0 = (i64)blockIdx.x * 256, k0 = (i64)blockIdx.y * 256;
    // lane = row k0 + 32 warp + lane; a[g] = its 32 bits of columns j0 + 32 g ...
    const u32 *in32 = reinterpret_cast<const u32 *>(in);
    const i64 k = k0 + 32 * warp + lane;
    u32 a[8];
#pragma unroll
    for (int g = 0; g < 8; ++g) {
        const i64 c = j0 + 32 * g;  // first column of word g
        u32 v = 0;
        if (k < kbits && c < cols) {
            v = in32[k * 2 * ld + (c >> 5)];
            if (cols - c < 32) v &= (1u << (cols - c)) - 1u;
        }
        a[g] = v;
    }
    // 32 x 32 bit transposes across the warp: afterwards lane l's a[g] holds,
    // at bit r, row k0 + 32 warp + r of column j0 + 32 g + l
#pragma unroll
    for (int g = 0; g < 8; ++g) a[g] = transpose32_warp(a[g]);
#pragma unroll
    for (int g = 0; g < 8; ++g) U[32 * g + lane][warp] = a[g];
    __syncthreads();
    if (F4) {
        // column j, k slice q (32 values): 16 bytes, value k in nibble k & 1 of byte k / 2
        for (int e = tid; e < 256 * 8; e += 256) {
            const int j = e >> 3, q = e & 7;
            const i64 kb = (k0 + 32 * q) / 2;  // byte offset in the output row
            if (kb >= kpad) continue;
            const u32 v = U[j][q];
            u32 o[4];
#pragma unroll
            for (int h = 0; h < 4; ++h) {
                const u32 x = (v >> (8 * h)) & 0xFFu;
                o[h] = (spread_even4(x & 0x55u) << 1) | (spread_even4((x >> 1) & 0x55u) << 5);
            }
            *reinterpret_cast<uint4 *>(out + (j0 + j) * kpad + kb) = make_uint4(o[0], o[1], o[2], o[3]);
        }
    } else {
        // column j, k slice q (16 values): 16 bytes of 0/1
        for (int e = tid; e < 256 * 16; e += 256) {
            const int j = e >> 4, q = e & 15;
            const i64 kb = k0 + 16 * q;
            if (kb >= kpad) continue;
            const u32 h = (U[j][q >> 1] >> (16 * (q & 1))) & 0xFFFFu;
            *reinterpret_cast<uint4 *>(out + (j0 + j) * kpad + kb) =
                make_uint4(spread4(h & 15), spread4((h >> 4) & 15), spread4((h >> 8) & 15), spread4((h >> 12) & 15));
        }
    }
}

// ---------------------------------------------------------------- launchers
static int grid_for(i64 total, int threads)
{
    i64 g = (total + threads - 1) / threads;
    i64 cap = (i64)sm_count() * 16;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

mela_status launch_expand_u8(const u64 *in, i64 ld, i64 rows, i64 kbits, i64 rows_pad, i64 kpad,
                             unsigned char *out, cudaStream_t s)
{
    i64 total = rows_pad * (kpad >> 6);
    expand_u8_kernel<<<grid_for(total, 256), 256, 0, s>>>(in, ld, rows, kbits, rows_pad, kpad, out);
    MELA_LAUNCH_CHECK("expand_u8_kernel");
    return MELA_OK;
}

mela_status launch_expand_f4(const u64 *in, i64 ld, i64 rows, i64 kbits, i64 rows_pad, i64 kpad_bytes,
                             unsigned char *out, cudaStream_t s)
{
    i64 total = rows_pad * (kpad_bytes >> 5);
    expand_f4_kernel<<<grid_for(total, 256), 256, 0, s>>>(in, ld, rows, kbits, rows_pad, kpad_bytes, out);
    MELA_LAUNCH_CHECK("expand_f4_kernel");
    return MELA_OK;
}

mela_status launch_expand_t(const u64 *in, i64 ld, i64 kbits, i64 cols, i64 cols_pad, i64 kpad,
                            unsigned char *out, bool fp4, cudaStream_t s)
{
    if (cols_pad <= 0 || kpad <= 0) return MELA_OK;
    if (cols_pad % 256) {
        set_error("expand_t: padded column count %lld is not a multiple of 256", cols_pad);
        return MELA_ERR_INVALID;
    }
    const i64 kvals = fp4 ? 2 * kpad : kpad;
    if (mela_status st = check_grid_yz((kvals + 255) / 256, 1, "expand_t"); st != MELA_OK) return st;
    dim3 grid((unsigned)(cols_pad / 256), (unsigned)((kvals + 255) / 256));
    if (fp4)
        expand_t_kernel<true><<<grid, 256, 0, s>>>(in, ld, kbits, cols, kpad, out);
    else
        expand_t_kernel<false><<<grid, 256, 0, s>>>(in, ld, kbits, cols, kpad, out);
    MELA_LAUNCH_CHECK("expand_t_kernel");
    return MELA_OK;
}

mela_status launch_transpose(const u64 *in, i64 ld_in, i64 rows, i64 cols, u64 *out, i64 ld_out,
                             cudaStream_t s)
{
    if (rows <= 0 || cols <= 0) return MELA_OK;
    if (mela_status st = check_grid_yz((rows + 255) / 256, 1, "transpose"); st != MELA_OK) return st;
    dim3 grid((unsigned)words_of(cols), (unsigned)((rows + 255) / 256));
    transpose_kernel<<<grid, 256, 0, s>>>(in, ld_in, rows, cols, out, ld_out);
    MELA_LAUNCH_CHECK("transpose_kernel");
    return MELA_OK;
}

mela_status launch_pack(int kind, i64 m, i64 n, const void *in, u64 *out, i64 ld, cudaStream_t s)
{
    return launch_pack_words(kind, m, n, in, out, ld, ld, s);
}

mela_status launch_pack_words(int kind, i64 m, i64 n, const void *in, u64 *out, i64 ld, i64 out_words,
                              cudaStream_t s)
{
    if (m <= 0) return MELA_OK;
    i64 wgroups = (out_words + 7) / 8;
    if (wgroups == 0) return MELA_OK;
    if (mela_status st = check_grid_yz(wgroups, 1, "pack"); st != MELA_OK) return st;
    dim3 grid((unsigned)((m + 31) / 32), (unsigned)wgroups);
    if (kind == MELA_KIND_DOUBLE)
        pack_kernel<double><<<grid, 256, 0, s>>>((const double *)in, m, n, out, ld, out_words);
    else
        pack_kernel<unsigned char><<<grid, 256, 0, s>>>((const unsigned char *)in, m, n, out, ld, out_words);
    MELA_LAUNCH_CHECK("pack_kernel");
    return MELA_OK;
}

mela_status launch_unpack(const u64 *in, i64 ld, i64 m, i64 n, unsigned char *out, cudaStream_t s)
{
    if (m <= 0 || n <= 0) return MELA_OK;
    if (mela_status st = check_grid_yz((words_of(n) + 7) / 8, 1, "unpack"); st != MELA_OK) return st;
    dim3 grid((unsigned)((m + 31) / 32), (unsigned)((words_of(n) + 7) / 8));
    unpack_kernel<<<grid, 256, 0, s>>>(in, ld, m, n, out);
    MELA_LAUNCH_CHECK("unpack_kernel");
    return MELA_OK;
}

mela_status launch_rand_bernoulli(u64 seed, u64 stream_id, i64 m, i64 n, double density, u64 *out,
                                  i64 ld, cudaStream_t s)
{
    if (m <= 0 || ld <= 0) return MELA_OK;
    double t = density * 65536.0;
    unsigned thresh = t <= 0 ? 0u : (t >= 65536.0 ? 65536u : (unsigned)t);
    rand_bernoulli_kernel<<<grid_for(m * ld, 256), 256, 0, s>>>(stream_key(seed, stream_id), m, n, thresh,
                                                                 out, ld);
    MELA_LAUNCH_CHECK("rand_bernoulli_kernel");
    return MELA_OK;
}

mela_status launch_rand_dense(u64 seed, u64 stream_id, i64 m, i64 n, u64 *out, i64 ld,
                              cudaStream_t s)
{
    if (m <= 0 || ld <= 0) return MELA_OK;
    rand_dense_kernel<<<grid_for(m * ld, 256), 256, 0, s>>>(stream_key(seed, stream_id), m, n,
                                                            words_of(n), out, ld);
    MELA_LAUNCH_CHECK("rand_dense_kernel");
    return MELA_OK;
}

}  // namespace mela

// ---------------------------------------------------------------- C ABI
using namespace mela;

extern "C" mela_status mela_dev_rand_dense(uint64_t seed, uint64_t stream_id, int64_t m,
                                           int64_t n, uint64_t *d_out, int64_t ld, void *stream)
{
    if (m < 0 || n < 0 || ld < words_of(n) || (m > 0 && ld > 0 && !d_out)) {
        set_error("mela_dev_rand_dense: bad shape or pointer");
        return MELA_ERR_INVALID;
    }
    return launch_rand_dense(seed, stream_id, m, n, (u64 *)d_out, ld, (cudaStream_t)stream);
}

extern "C" mela_status mela_dev_rand_bernoulli(uint64_t seed, uint64_t stream_id, int64_t m,
                                               int64_t n, double density, uint64_t *d_out, int64_t ld,
                                               void *stream)
{
    if (m < 0 || n < 0 || ld < words_of(n) || (m > 0 && ld > 0 && !d_out) || !(density >= 0.0)) {
        set_error("mela_dev_rand_bernoulli: bad shape, pointer or density");
        return MELA_ERR_INVALID;
    }
    return launch_rand_bernoulli(seed, stream_id, m, n, density, (u64 *)d_out, ld, (cudaStream_t)stream);
}

extern "C" mela_status mela_dev_pack(int32_t kind, int64_t m, int64_t n, const void *d_in,
                                     uint64_t *d_out, int64_t ld, void *stream)
{
    if (m < 0 || n < 0 || ld < words_of(n) || (kind != MELA_KIND_LOGICAL && kind != MELA_KIND_DOUBLE)) {
        set_error("mela_dev_pack: bad shape or kind");
        return MELA_ERR_INVALID;
    }
    if (m > 0 && ld > 0 && (!d_out || (n > 0 && !d_in))) {
        set_error("mela_dev_pack: null pointer");
        return MELA_ERR_INVALID;
    }
    return launch_pack(kind, m, n, d_in, (u64 *)d_out, ld, (cudaStream_t)stream);
}

extern "C" mela_status mela_dev_unpack(const uint64_t *d_in, int64_t ld, int64_t m, int64_t n,
                                       uint8_t *d_out, void *stream)
{
    if (m < 0 || n < 0 || ld < words_of(n) || (m > 0 && n > 0 && (!d_in || !d_out))) {
        set_error("mela_dev_unpack: bad shape or pointer");
        return MELA_ERR_INVALID;
    }
    return launch_unpack((const u64 *)d_in, ld, m, n, d_out, (cudaStream_t)stream);
}

extern "C" mela_status mela_dev_transpose(const uint64_t *d_in, int64_t ld_in, int64_t rows,
                                          int64_t cols, uint64_t *d_out, int64_t ld_out,
                                          void *stream)
{
    if (rows < 0 || cols < 0 || ld_in < words_of(cols) || ld_out < words_of(rows) ||
        (rows > 0 && cols > 0 && (!d_in || !d_out))) {
        set_error("mela_dev_transpose: bad shape or pointer");
        return MELA_ERR_INVALID;
    }
    return launch_transpose((const u64 *)d_in, ld_in, rows, cols, (u64 *)d_out, ld_out,
                            (cudaStream_t)stream);
}
