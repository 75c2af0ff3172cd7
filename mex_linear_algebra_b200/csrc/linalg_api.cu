// linalg_api.cu -- C ABI for rank, reduced row echelon form and null space.
//
// Host entry points take a MATLAB-layout matrix, run everything on the GPU
// (pack, eliminate, extract the basis, unpack) and copy the result back.
// Device entry points are stream-ordered on packed matrices.
#include <algorithm>

#include "mela_common.cuh"
#include "mela_internal.h"
#include "mela_host.h"
#include "elim.h"

namespace mela {

static bool ok_kind(int k) { return k == MELA_KIND_LOGICAL || k == MELA_KIND_DOUBLE; }

// Rank of a packed device matrix (overwritten), read back to the host.
mela_status rank_of_packed(u64 *P, i64 ld, i64 m, i64 n, int variant, cudaStream_t s, double *rank)
{
    const i64 mn = m < n ? m : n;
    DevBuf ws, out;
    mela_status st;
    const size_t wsb = elim_workspace(m, n);
    if ((st = ws.alloc(wsb, s)) != MELA_OK) return st;
    if ((st = out.alloc((size_t)(1 + 2 * mn) * 8, s)) != MELA_OK) return st;
    long long *d = (long long *)out.p;
    st = elim_device(variant, P, ld, m, n, 0, d, d + 1, d + 1 + mn, ws.p, wsb, s);
    if (st != MELA_OK) return st;
    long long r = 0;
    MELA_CUDA_TRY(cudaMemcpyAsync(&r, d, sizeof r, cudaMemcpyDeviceToHost, s));
    if ((st = finish(s)) != MELA_OK) return st;
    *rank = (double)r;
    return MELA_OK;
}

// Null-space basis of a packed device matrix (overwritten by its RREF) into
// the caller's n x nullity logical buffer from `alloc`.  m may be 0.
mela_status null_of_packed(u64 *P, i64 ld, i64 m, i64 n, int variant, mela_alloc_fn alloc, void *ctx,
                           int64_t *nullity, cudaStream_t s)
{
    if (n == 0) {
        if (nullity) *nullity = 0;
        alloc(ctx, 0, 0);  // an empty n x 0 result; the buffer is not written
        return MELA_OK;
    }
    const i64 mn = m < n ? m : n;
    mela_status st;
    DevBuf ws, out;
    if ((st = out.alloc((size_t)(1 + 2 * (mn ? mn : 1)) * 8, s)) != MELA_OK) return st;
    long long *d = (long long *)out.p;
    long long r = 0;
    if (m > 0) {
        const size_t wsb = elim_workspace(m, n);
        if ((st = ws.alloc(wsb, s)) != MELA_OK) return st;
        st = elim_device(variant, P, ld, m, n, 1, d, d + 1, d + 1 + mn, ws.p, wsb, s);
        if (st != MELA_OK) return st;
        MELA_CUDA_TRY(cudaMemcpyAsync(&r, d, sizeof r, cudaMemcpyDeviceToHost, s));
        MELA_CUDA_TRY(cudaStreamSynchronize(s));
    }
    const i64 f = n - r;
    uint8_t *Z = alloc(ctx, n, f);
    if (!Z && f > 0) {
        set_error("output allocation failed");
        return MELA_ERR_NOMEM;
    }
    if (nullity) *nullity = f;
    if (f == 0) return finish(s);
    const i64 ldz = even_words(n);
    DevBuf Zt, nws, bytes;
    if ((st = Zt.alloc((size_t)f * ldz * 8, s)) != MELA_OK) return st;
    const NullLayout NL = null_layout(n, r);
    if ((st = nws.alloc(NL.total, s)) != MELA_OK) return st;
    st = null_basis_device((const u64 *)P, ld, m, n, r, d + 1, d + 1 + mn, (u64 *)Zt.p, ldz, nws.p, NL.total, s);
    if (st != MELA_OK) return st;
    if ((st = bytes.alloc((size_t)f * n, s)) != MELA_OK) return st;
    if ((st = launch_unpack_rows((const u64 *)Zt.p, ldz, f, n, (unsigned char *)bytes.p, s)) != MELA_OK)
        return st;
    MELA_CUDA_TRY(cudaMemcpyAsync(Z, bytes.p, (size_t)f * n, cudaMemcpyDeviceToHost, s));
    return finish(s);
}

mela_status host_rank(const mela_host_matrix *A, int variant, double *rank)
{
    if (!A || !rank) {
        set_error("null argument");
        return MELA_ERR_INVALID;
    }
    if (!ok_kind(A->kind)) return MELA_ERR_TYPE;
    const i64 m = A->rows, n = A->cols;
    if (m < 0 || n < 0) return MELA_ERR_INVALID;
    if (m == 0 || n == 0) {
        *rank = 0.0;
        return MELA_OK;
    }
    if (!A->data) {
        set_error("null data pointer");
        return MELA_ERR_INVALID;
    }
    cudaStream_t s;
    mela_status st = host_stream(&s);
    if (st != MELA_OK) return st;
    const i64 ld = even_words(n);
    DevBuf P, stage;
    if ((st = P.alloc((size_t)m * ld * 8, s)) != MELA_OK) return st;
    if ((st = upload_and_pack(A, (u64 *)P.p, ld, s, stage)) != MELA_OK) return st;
    return rank_of_packed((u64 *)P.p, ld, m, n, variant, s, rank);
}

mela_status host_null(const mela_host_matrix *H, int variant, mela_alloc_fn alloc, void *ctx,
                      int64_t *nullity)
{
    if (!H || !alloc) {
        set_error("null argument");
        return MELA_ERR_INVALID;
    }
    if (H->sparse) return MELA_ERR_SPARSE;
    if (!ok_kind(H->kind)) return MELA_ERR_TYPE;
    const i64 m = H->rows, n = H->cols;
    if (m < 0 || n < 0) return MELA_ERR_INVALID;
    if (n == 0) {
        if (nullity) *nullity = 0;
        alloc(ctx, 0, 0);  // an empty n x 0 result; the buffer is not written
        return MELA_OK;
    }
    if (m > 0 && !H->data) {
        set_error("null data pointer");
        return MELA_ERR_INVALID;
    }
    cudaStream_t s;
    mela_status st = host_stream(&s);
    if (st != MELA_OK) return st;
    const i64 ld = even_words(n);
    DevBuf P, stage;
    if ((st = P.alloc((size_t)(m ? m : 1) * ld * 8, s)) != MELA_OK) return st;
    if (m > 0 && (st = upload_and_pack(H, (u64 *)P.p, ld, s, stage)) != MELA_OK) return st;
    return null_of_packed((u64 *)P.p, ld, m, n, variant, alloc, ctx, nullity, s);
}

// Rows of C (rows x w words) with any nonzero word, added to *count.
__global__ void count_nonzero_rows_kernel(const u64 *__restrict__ C, i64 ldc, i64 rows, i64 w,
                                          long long *count)
{
    long long mine = 0;
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < rows; i += (i64)gridDim.x * blockDim.x) {
        u64 any = 0;
        for (i64 x = 0; x < w; ++x) any |= C[i * ldc + x];
        mine += any != 0;
    }
    mine = __reduce_add_sync(0xffffffffu, (unsigned)mine);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd((unsigned long long *)count, (unsigned long long)mine);
}

}  // namespace mela

using namespace mela;

// ---------------------------------------------------------------- host ABI
extern "C" mela_status mela_rank_gf2(const mela_host_matrix *A, double *rank)
{
    return host_rank(A, MELA_ELIM_AUTO, rank);
}

extern "C" mela_status mela_rank_m4ri(const mela_host_matrix *A, double *rank)
{
    return host_rank(A, MELA_ELIM_M4RI, rank);
}

extern "C" mela_status mela_null_gf2(const mela_host_matrix *H, mela_alloc_fn alloc, void *ctx,
                                     int64_t *nullity)
{
    return host_null(H, MELA_ELIM_AUTO, alloc, ctx, nullity);
}

extern "C" mela_status mela_null_m4ri(const mela_host_matrix *H, mela_alloc_fn alloc, void *ctx,
                                      int64_t *nullity)
{
    return host_null(H, MELA_ELIM_M4RI, alloc, ctx, nullity);
}

// ---------------------------------------------------------------- device ABI
extern "C" size_t mela_elim_workspace_size(int64_t m, int64_t n)
{
    if (m <= 0 || n <= 0) return 0;
    return elim_workspace(m, n);
}

static mela_status check_elim(int32_t variant, const uint64_t *dM, int64_t ld, int64_t m, int64_t n)
{
    Tuning t;
    if (m < 0 || n < 0 || ld < words_of(n) || !decode_elim_variant(variant, &t)) {
        set_error("bad shape, leading dimension or variant");
        return MELA_ERR_INVALID;
    }
    if (m > 0 && n > 0 && !dM) {
        set_error("null matrix");
        return MELA_ERR_INVALID;
    }
    return MELA_OK;
}

extern "C" mela_status mela_dev_rank(int32_t variant, uint64_t *dM, int64_t ld, int64_t m, int64_t n,
                                     int64_t *d_rank, int64_t *d_pivcols, int64_t *d_pivrows,
                                     void *workspace, size_t workspace_bytes, void *stream)
{
    mela_status st = check_elim(variant, dM, ld, m, n);
    if (st != MELA_OK) return st;
    if (!d_rank || (m > 0 && n > 0 && (!d_pivcols || !d_pivrows))) {
        set_error("null output");
        return MELA_ERR_INVALID;
    }
    return elim_device(variant, (u64 *)dM, ld, m, n, 0, (long long *)d_rank, (long long *)d_pivcols,
                       (long long *)d_pivrows, workspace, workspace_bytes, (cudaStream_t)stream);
}

extern "C" mela_status mela_dev_rref(int32_t variant, uint64_t *dM, int64_t ld, int64_t m, int64_t n,
                                     int64_t *d_rank, int64_t *d_pivcols, int64_t *d_pivrows,
                                     void *workspace, size_t workspace_bytes, void *stream)
{
    mela_status st = check_elim(variant, dM, ld, m, n);
    if (st != MELA_OK) return st;
    if (!d_rank || (m > 0 && n > 0 && (!d_pivcols || !d_pivrows))) {
        set_error("null output");
        return MELA_ERR_INVALID;
    }
    return elim_device(variant, (u64 *)dM, ld, m, n, 1, (long long *)d_rank, (long long *)d_pivcols,
                       (long long *)d_pivrows, workspace, workspace_bytes, (cudaStream_t)stream);
}

extern "C" size_t mela_null_workspace_size(int64_t n, int64_t rank)
{
    if (n <= 0 || rank < 0 || rank > n) return 0;
    return null_layout(n, rank).total;
}

extern "C" mela_status mela_dev_null_basis(const uint64_t *dR, int64_t ld, int64_t m, int64_t n,
                                           int64_t rank, const int64_t *d_pivcols,
                                           const int64_t *d_pivrows, uint64_t *dZt, int64_t ldz,
                                           void *workspace, size_t workspace_bytes, void *stream)
{
    if (m < 0 || n < 0 || rank < 0 || rank > n || rank > m || ld < words_of(n) || ldz < words_of(n)) {
        set_error("mela_dev_null_basis: bad shape");
        return MELA_ERR_INVALID;
    }
    if (n - rank > 0 && (!dZt || (rank > 0 && (!dR || !d_pivcols || !d_pivrows)))) {
        set_error("mela_dev_null_basis: null pointer");
        return MELA_ERR_INVALID;
    }
    return null_basis_device((const u64 *)dR, ld, m, n, rank, (const long long *)d_pivcols,
                             (const long long *)d_pivrows, (u64 *)dZt, ldz, workspace, workspace_bytes,
                             (cudaStream_t)stream);
}

extern "C" mela_status mela_dev_unpack_rows(const uint64_t *d_in, int64_t ld, int64_t rows, int64_t n,
                                            uint8_t *d_out, void *stream)
{
    if (rows < 0 || n < 0 || ld < words_of(n) || (rows > 0 && n > 0 && (!d_in || !d_out))) {
        set_error("mela_dev_unpack_rows: bad shape or pointer");
        return MELA_ERR_INVALID;
    }
    return launch_unpack_rows((const u64 *)d_in, ld, rows, n, d_out, (cudaStream_t)stream);
}

extern "C" size_t mela_null_verify_workspace_size(int64_t m, int64_t f)
{
    if (m <= 0 || f <= 0) return 0;
    return (size_t)m * (size_t)words_of(f) * 8;
}

extern "C" mela_status mela_dev_null_verify(const uint64_t *dA, int64_t lda, int64_t m, int64_t n,
                                            const uint64_t *dZt, int64_t ldz, int64_t f,
                                            int64_t *d_bad_rows, void *workspace, size_t workspace_bytes,
                                            void *stream)
{
    if (m < 0 || n < 0 || f < 0 || lda < words_of(n) || ldz < words_of(n)) {
        set_error("mela_dev_null_verify: bad shape");
        return MELA_ERR_INVALID;
    }
    if (!d_bad_rows || (m > 0 && n > 0 && f > 0 && (!dA || !dZt))) {
        set_error("mela_dev_null_verify: null pointer");
        return MELA_ERR_INVALID;
    }
    const size_t need = mela_null_verify_workspace_size(m, f);
    if (workspace_bytes < need || (need && !workspace)) {
        set_error("mela_dev_null_verify: workspace of %zu bytes needed, %zu given", need, workspace_bytes);
        return MELA_ERR_INVALID;
    }
    const cudaStream_t s = (cudaStream_t)stream;
    MELA_CUDA_TRY(cudaMemsetAsync(d_bad_rows, 0, sizeof(int64_t), s));
    if (m == 0 || f == 0) return MELA_OK;
    // C (m x f) = A (m x n) * Z (n x f); the plain product takes Z^T = Zt as is
    u64 *C = (u64 *)workspace;
    const i64 wf = words_of(f);
    mela_status st = launch_gemm_plain((const u64 *)dA, lda, (const u64 *)dZt, ldz, C, wf, m, n, f, s);
    if (st != MELA_OK) return st;
    const i64 blocks = std::min<i64>((m + 255) / 256, (i64)4 * sm_count());
    count_nonzero_rows_kernel<<<(unsigned)blocks, 256, 0, s>>>(C, wf, m, wf, (long long *)d_bad_rows);
    MELA_LAUNCH_CHECK("count_nonzero_rows_kernel");
    return MELA_OK;
}
