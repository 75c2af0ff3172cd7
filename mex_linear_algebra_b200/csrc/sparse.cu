// sparse.cu -- compressed-sparse-column input packed on the GPU.
//
// No counterpart in the reference, whose gateways reject sparse arrays
// (src/mela_matmul_gf2.c:78-79, src/mela_null_gf2.c:150) or, for the rank
// functions, read their value array as if it were dense.  Parity-check
// matrices are naturally sparse (a few ones per row), so the library takes
// MATLAB's own sparse layout directly: column j holds the entries
// colptr[j] .. colptr[j+1]-1 with rows rowidx[e] (0-based, 64-bit: MATLAB's
// jc / ir), and optional values (logical bytes or doubles, a double read as
// ((int)x) & 1 like dense input).  Repeated (row, column) entries add mod 2.
#include <climits>
#include <cmath>

#include "mela_common.cuh"
#include "mela_internal.h"
#include "mela_host.h"
#include "elim.h"

namespace mela {

__device__ __forceinline__ bool csc_bit(int kind, const void *values, i64 e)
{
    if (!values) return true;
    if (kind == MELA_KIND_DOUBLE) {
        const double x = static_cast<const double *>(values)[e];
        // ((int)x) & 1; NaN and values outside the int range read as 0
        if (!(x > -2147483649.0 && x < 2147483648.0)) return false;
        return ((int)x) & 1;
    }
    return static_cast<const unsigned char *>(values)[e] & 1;
}

// A warp per column, lanes over its entries; each set entry flips its bit
// in the (zeroed) packed output.  Row indices outside [0, m) are skipped and
// reported through the device error word.
__global__ void pack_csc_kernel(const long long *__restrict__ colptr, const long long *__restrict__ rowidx,
                                const void *values, int kind, i64 m, i64 n, u64 *__restrict__ out, i64 ld,
                                u32 *err)
{
    const int lane = threadIdx.x & 31;
    const i64 wpb = blockDim.x >> 5;
    for (i64 j = blockIdx.x * wpb + (threadIdx.x >> 5); j < n; j += (i64)gridDim.x * wpb) {
        const i64 e0 = colptr[j], e1 = colptr[j + 1];
        const u64 bit = 1ull << (j & 63);
        const i64 wj = j >> 6;
        for (i64 e = e0 + lane; e < e1; e += 32) {
            const i64 i = rowidx[e];
            if (i < 0 || i >= m) {
                atomicOr(err, kErrBadArgument);
                continue;
            }
            if (csc_bit(kind, values, e)) atomicXor(&out[i * ld + wj], bit);
        }
    }
}

mela_status launch_pack_csc(const long long *colptr, const long long *rowidx, const void *values, int kind, i64 m,
                            i64 n, u64 *out, i64 ld, cudaStream_t s)
{
    if (m <= 0 || n <= 0) return MELA_OK;
    MELA_CUDA_TRY(cudaMemsetAsync(out, 0, (size_t)m * ld * 8, s));
    i64 blocks = (n + 7) / 8;  // 8 warps per block
    const i64 cap = (i64)sm_count() * 16;
    if (blocks > cap) blocks = cap;
    pack_csc_kernel<<<(unsigned)blocks, 256, 0, s>>>(colptr, rowidx, values, kind, m, n, out, ld,
                                                     device_error_word());
    MELA_LAUNCH_CHECK("pack_csc_kernel");
    return MELA_OK;
}

// Host CSC -> packed device matrix (checked on the host first: column
// pointers from 0, non-decreasing; every row index in range).
static mela_status upload_csc(const mela_host_csc *H, u64 *dP, i64 ld, cudaStream_t s, DevBuf &cp, DevBuf &ri,
                              DevBuf &va)
{
    const i64 m = H->rows, n = H->cols;
    const i64 nnz = H->colptr[n];
    mela_status st;
    if ((st = cp.alloc((size_t)(n + 1) * 8, s)) != MELA_OK) return st;
    MELA_CUDA_TRY(cudaMemcpyAsync(cp.p, H->colptr, (size_t)(n + 1) * 8, cudaMemcpyHostToDevice, s));
    if ((st = ri.alloc((size_t)(nnz ? nnz : 1) * 8, s)) != MELA_OK) return st;
    if (nnz) MELA_CUDA_TRY(cudaMemcpyAsync(ri.p, H->rowidx, (size_t)nnz * 8, cudaMemcpyHostToDevice, s));
    const void *dv = nullptr;
    if (H->values && nnz) {
        const size_t esz = H->kind == MELA_KIND_DOUBLE ? 8 : 1;
        if ((st = va.alloc((size_t)nnz * esz, s)) != MELA_OK) return st;
        MELA_CUDA_TRY(cudaMemcpyAsync(va.p, H->values, (size_t)nnz * esz, cudaMemcpyHostToDevice, s));
        dv = va.p;
    }
    return launch_pack_csc((const long long *)cp.p, (const long long *)ri.p, dv, H->kind, m, n, dP, ld, s);
}

static mela_status check_csc(const mela_host_csc *H)
{
    if (!H) {
        set_error("null argument");
        return MELA_ERR_INVALID;
    }
    if (H->rows < 0 || H->cols < 0 || H->rows > INT_MAX - 1) {
        set_error("bad sparse matrix shape");
        return MELA_ERR_INVALID;
    }
    if (H->values && H->kind != MELA_KIND_LOGICAL && H->kind != MELA_KIND_DOUBLE) return MELA_ERR_TYPE;
    if (!H->colptr) {
        set_error("null column pointers");
        return MELA_ERR_INVALID;
    }
    if (H->colptr[0] != 0) {
        set_error("column pointers must start at 0");
        return MELA_ERR_INVALID;
    }
    for (i64 j = 0; j < H->cols; ++j)
        if (H->colptr[j + 1] < H->colptr[j]) {
            set_error("column pointers must not decrease (column %lld)", (long long)j);
            return MELA_ERR_INVALID;
        }
    const i64 nnz = H->colptr[H->cols];
    if (nnz > 0 && !H->rowidx) {
        set_error("null row indices");
        return MELA_ERR_INVALID;
    }
    for (i64 e = 0; e < nnz; ++e)
        if (H->rowidx[e] < 0 || H->rowidx[e] >= H->rows) {
            set_error("row index %lld of entry %lld outside [0, %lld)", (long long)H->rowidx[e], (long long)e,
                      (long long)H->rows);
            return MELA_ERR_INVALID;
        }
    return MELA_OK;
}

}  // namespace mela

using namespace mela;

extern "C" mela_status mela_dev_pack_csc(const int64_t *d_colptr, const int64_t *d_rowidx, const void *d_values,
                                         int32_t kind, int64_t m, int64_t n, uint64_t *d_out, int64_t ld,
                                         void *stream)
{
    if (m < 0 || n < 0 || ld < words_of(n) || (m > 0 && n > 0 && (!d_colptr || !d_out)) ||
        (d_values && kind != MELA_KIND_LOGICAL && kind != MELA_KIND_DOUBLE)) {
        set_error("mela_dev_pack_csc: bad arguments");
        return MELA_ERR_INVALID;
    }
    return launch_pack_csc((const long long *)d_colptr, (const long long *)d_rowidx, d_values, kind, m, n,
                           (u64 *)d_out, ld, (cudaStream_t)stream);
}

extern "C" mela_status mela_rank_csc(const mela_host_csc *H, int64_t *rank)
{
    mela_status st = check_csc(H);
    if (st != MELA_OK) return st;
    if (!rank) {
        set_error("null argument");
        return MELA_ERR_INVALID;
    }
    const i64 m = H->rows, n = H->cols;
    if (m == 0 || n == 0) {
        *rank = 0;
        return MELA_OK;
    }
    cudaStream_t s;
    if ((st = host_stream(&s)) != MELA_OK) return st;
    const i64 ld = even_words(n);
    DevBuf P, cp, ri, va;
    if ((st = P.alloc((size_t)m * ld * 8, s)) != MELA_OK) return st;
    if ((st = upload_csc(H, (u64 *)P.p, ld, s, cp, ri, va)) != MELA_OK) return st;
    double r = 0;
    if ((st = rank_of_packed((u64 *)P.p, ld, m, n, MELA_ELIM_AUTO, s, &r)) != MELA_OK) return st;
    *rank = (int64_t)r;
    return MELA_OK;
}

extern "C" mela_status mela_null_csc(const mela_host_csc *H, mela_alloc_fn alloc, void *ctx, int64_t *nullity)
{
    mela_status st = check_csc(H);
    if (st != MELA_OK) return st;
    if (!alloc) {
        set_error("null argument");
        return MELA_ERR_INVALID;
    }
    const i64 m = H->rows, n = H->cols;
    cudaStream_t s;
    if ((st = host_stream(&s)) != MELA_OK) return st;
    const i64 ld = even_words(n ? n : 1);
    DevBuf P, cp, ri, va;
    if ((st = P.alloc((size_t)(m ? m : 1) * ld * 8, s)) != MELA_OK) return st;
    if (m > 0 && n > 0 && (st = upload_csc(H, (u64 *)P.p, ld, s, cp, ri, va)) != MELA_OK) return st;
    return null_of_packed((u64 *)P.p, ld, m, n, MELA_ELIM_AUTO, alloc, ctx, nullity, s);
}
