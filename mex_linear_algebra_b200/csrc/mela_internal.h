// mela_internal.h -- launchers shared between the library's translation units.
#pragma once

#include <cuda.h>

#include "mela_common.cuh"

namespace mela {

u64 stream_key(u64 seed, u64 stream);

mela_status launch_rand_dense(u64 seed, u64 stream_id, i64 m, i64 n, u64 *out, i64 ld,
                              cudaStream_t s);
mela_status launch_rand_bernoulli(u64 seed, u64 stream_id, i64 m, i64 n, double density, u64 *out,
                                  i64 ld, cudaStream_t s);
mela_status launch_pack(int kind, i64 m, i64 n, const void *in, u64 *out, i64 ld, cudaStream_t s);
// The same, writing only the first out_words words of each packed row (the
// words of a column block, for packing a matrix block by block).
mela_status launch_pack_words(int kind, i64 m, i64 n, const void *in, u64 *out, i64 ld, i64 out_words,
                              cudaStream_t s);
mela_status launch_unpack(const u64 *in, i64 ld, i64 m, i64 n, unsigned char *out, cudaStream_t s);
mela_status launch_transpose(const u64 *in, i64 ld_in, i64 rows, i64 cols, u64 *out, i64 ld_out,
                             cudaStream_t s);
mela_status launch_expand_f4(const u64 *in, i64 ld, i64 rows, i64 kbits, i64 rows_pad, i64 kpad_bytes,
                             unsigned char *out, cudaStream_t s);
// Column j of the packed kbits x cols matrix `in` as row j of a K-major
// tensor-core operand (cols_pad rows, a multiple of 256; kpad bytes per row:
// 0/1 bytes, or e2m1 pairs when fp4), zero past kbits and cols.
mela_status launch_expand_t(const u64 *in, i64 ld, i64 kbits, i64 cols, i64 cols_pad, i64 kpad,
                            unsigned char *out, bool fp4, cudaStream_t s);
mela_status launch_expand_u8(const u64 *in, i64 ld, i64 rows, i64 kbits, i64 rows_pad, i64 kpad,
                             unsigned char *out, cudaStream_t s);

// ---- products (packed, device)
// Plain AND+popcount product: C (m x n) = A (m x k) * B (k x n), with the
// transposed right operand Bt (n x k) already formed.
mela_status launch_gemm_plain(const u64 *A, i64 lda, const u64 *Bt, i64 ldbt, u64 *C, i64 ldc,
                              i64 m, i64 k, i64 n, cudaStream_t s);
// Tensor-core product on 0/1 byte operands A8 (mp x kp) and Bt8 (np x kp),
// both K-major; mp % 128 == 0, np % 256 == 0, kp % 128 == 0.  Writes the
// valid m x n block of packed C.
// fp4 = true: packed e2m1 operands (kp counts bytes, two values each), kind::mxf4.
// tile: 0 = CTA pairs (256 x 256 tiles) when mp % 256 == 0, else one CTA per
// 128 x 256 tile; 1 = always one CTA per tile; 2 = pairs where mp allows.
mela_status launch_gemm_tc(const unsigned char *A8, const unsigned char *Bt8, i64 mp, i64 np,
                           i64 kp, u64 *C, i64 ldc, i64 m, i64 n, cudaStream_t s, bool fp4, int tile = 0);
// TMA map of a K-major byte matrix rows x kp (row pitch kp bytes): boxes of
// 128 bytes x box_rows rows with 128-byte swizzle, as the tcgen05 kernels read them.
mela_status make_u8_kmajor_map(CUtensorMap *map, const unsigned char *base, i64 rows, i64 kp, int box_rows);
// TMA map of packed rows (rows x words uint64, row pitch ld words; ld * 8 must
// be a multiple of 16 and base 16-byte aligned): boxes of box_words x box_rows,
// no swizzle, zeros read past the edges.
mela_status make_u64_rows_map(CUtensorMap *map, const u64 *base, i64 rows, i64 words, i64 ld, int box_words,
                              int box_rows);
// tile: 0 / 2 = 16 warps of 32 rows per 512-row CTA, 1 = 8 warps of 64 rows.
mela_status launch_gemm_m4ri(const u64 *A, i64 lda, const u64 *B, i64 ldb, u64 *C, i64 ldc,
                             i64 m, i64 k, i64 n, cudaStream_t s, int tile = 0);

// Whole RREF of one matrix in one single-CTA launch (batch.cu).
size_t fused_workspace(i64 m, i64 n);
mela_status launch_fused_elim(u64 *M, i64 ld, i64 m, i64 n, long long *d_rank, long long *d_piv,
                              long long *d_prow, void *ws, size_t ws_bytes, cudaStream_t s);

}  // namespace mela
