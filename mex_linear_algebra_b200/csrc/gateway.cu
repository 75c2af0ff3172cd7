// gateway.cu -- the MEX gateway semantics of the six reference functions, in
// one place, for the MATLAB gateways (mex/*.c) and for any other front end
// (the Python module uses it through ctypes).
//
// Argument checks run in the reference's order and fail with the
// reference's identifiers and messages:
//   products   src/mela_matmul_gf2.c:75-88, src/mela_matmul_m4ri.c:143-156
//   rank       src/mela_rank_gf2.c:128-133 (identifiers bitrank_mex:*),
//              src/mela_rank_m4ri.c:289-291, :331-334
//   null space src/mela_null_gf2.c:143-156, src/mela_null_m4ri.c:252-265
// Quirks kept: the rank functions do not reject sparse input or extra
// outputs; a zero-size packed matrix fails where the reference's zero-byte
// mxCalloc does (rank_gf2: "Unable to allocate memory for packed matrix.",
// null: "Out of memory."), while rank_m4ri (plain calloc) returns 0.
// Failures with no reference counterpart (CUDA errors, timeouts) use the
// identifier "mela:<status>".
#include <cstdio>
#include <cstring>

#include "mela_common.cuh"
#include "mela_internal.h"
#include "mela_host.h"

namespace {

struct Out {
    mela_gateway_alloc_fn alloc;
    void *ctx;
};

void fail(mela_gateway_error *err, const char *id, const char *msg)
{
    if (!err) return;
    snprintf(err->id, sizeof err->id, "%s", id);
    snprintf(err->msg, sizeof err->msg, "%s", msg);
}

int fail_status(mela_gateway_error *err, const char *fn, mela_status st)
{
    char id[64], msg[256];
    snprintf(id, sizeof id, "mela:%s", mela_status_string(st));
    for (char *c = id; *c; ++c)
        if (*c == ' ') *c = '_';
    snprintf(msg, sizeof msg, "%s: %s: %s", fn, mela_status_string(st), mela_last_error());
    fail(err, id, msg);
    return 1;
}

bool is_ld(int32_t k) { return k == MELA_KIND_LOGICAL || k == MELA_KIND_DOUBLE; }

struct NullCtx {
    Out out;
    uint8_t *buf;
};

uint8_t *null_alloc(void *c, int64_t rows, int64_t cols)
{
    NullCtx *x = (NullCtx *)c;
    x->buf = (uint8_t *)x->out.alloc(x->out.ctx, 0, MELA_KIND_LOGICAL, rows, cols);
    return x->buf;
}

}  // namespace

extern "C" int mela_gateway(int32_t fn, int32_t nlhs, int32_t nrhs, const mela_host_matrix *prhs,
                            mela_gateway_alloc_fn alloc, void *ctx, mela_gateway_error *err)
{
    if (err) {
        err->id[0] = 0;
        err->msg[0] = 0;
    }
    if (!alloc) {
        fail(err, "mela:invalid", "no output allocator");
        return 1;
    }
    switch (fn) {
    case MELA_FN_MATMUL_GF2:
    case MELA_FN_MATMUL_M4RI: {
        const char *name = fn == MELA_FN_MATMUL_GF2 ? "mela_matmul_gf2" : "mela_matmul_m4ri";
        if (nrhs != 2) return fail(err, "", "Need two input matrices A,B."), 1;
        if (nlhs > 1) return fail(err, "", "Too many outputs."), 1;
        const mela_host_matrix *A = &prhs[0], *B = &prhs[1];
        if (A->sparse || B->sparse)
            return fail(err, "", "Sparse matrices not supported. Convert to full using full()."), 1;
        if (A->cols != B->rows) return fail(err, "", "Inner dimensions must agree."), 1;
        if (!is_ld(A->kind) || !is_ld(B->kind))
            return fail(err, "", "Inputs must be logical or double matrices."), 1;
        uint8_t *C = (uint8_t *)alloc(ctx, 0, MELA_KIND_LOGICAL, A->rows, B->cols);
        if (!C && A->rows * B->cols > 0) return fail_status(err, name, MELA_ERR_NOMEM);
        const mela_status st = fn == MELA_FN_MATMUL_GF2 ? mela_matmul_gf2(A, B, C) : mela_matmul_m4ri(A, B, C);
        if (st != MELA_OK) return fail_status(err, name, st);
        return 0;
    }
    case MELA_FN_RANK_GF2: {
        if (nrhs != 1) return fail(err, "bitrank_mex:nargin", "One input required."), 1;
        const mela_host_matrix *A = &prhs[0];
        if (!is_ld(A->kind))
            return fail(err, "bitrank_mex:inputNotLogical", "Input must be a logical or double matrix."), 1;
        if (A->rows * ((A->cols + 63) / 64) == 0)
            return fail(err, "bitrank_mex:memory", "Unable to allocate memory for packed matrix."), 1;
        double *r = (double *)alloc(ctx, 0, MELA_KIND_DOUBLE, 1, 1);
        if (!r) return fail_status(err, "mela_rank_gf2", MELA_ERR_NOMEM);
        mela_host_matrix dense = *A;
        dense.sparse = 0;
        const mela_status st = mela_rank_gf2(&dense, r);
        if (st != MELA_OK) return fail_status(err, "mela_rank_gf2", st);
        return 0;
    }
    case MELA_FN_RANK_M4RI: {
        if (nrhs != 1) return fail(err, "", "One input required."), 1;
        const mela_host_matrix *A = &prhs[0];
        if (!is_ld(A->kind)) return fail(err, "", "Input must be double or logical."), 1;
        double *r = (double *)alloc(ctx, 0, MELA_KIND_DOUBLE, 1, 1);
        if (!r) return fail_status(err, "mela_rank_m4ri", MELA_ERR_NOMEM);
        mela_host_matrix dense = *A;
        dense.sparse = 0;
        const mela_status st = mela_rank_m4ri(&dense, r);
        if (st != MELA_OK) return fail_status(err, "mela_rank_m4ri", st);
        return 0;
    }
    case MELA_FN_NULL_GF2:
    case MELA_FN_NULL_M4RI: {
        const char *name = fn == MELA_FN_NULL_GF2 ? "mela_null_gf2" : "mela_null_m4ri";
        if (nrhs != 1) return fail(err, "", "One input required: H."), 1;
        if (nlhs > 1) return fail(err, "", "One output required."), 1;
        const mela_host_matrix *H = &prhs[0];
        if (H->sparse)
            return fail(err, "", "Sparse matrices not supported. Convert to full using full()."), 1;
        if (!is_ld(H->kind)) return fail(err, "", "H must be double or logical."), 1;
        if (H->rows * ((H->cols + 63) / 64) == 0) return fail(err, "", "Out of memory."), 1;
        NullCtx c{{alloc, ctx}, nullptr};
        int64_t f = 0;
        const mela_status st = fn == MELA_FN_NULL_GF2 ? mela_null_gf2(H, null_alloc, &c, &f)
                                                      : mela_null_m4ri(H, null_alloc, &c, &f);
        if (st != MELA_OK) return fail_status(err, name, st);
        return 0;
    }
    default:
        fail(err, "mela:invalid", "unknown gateway function");
        return 1;
    }
}
