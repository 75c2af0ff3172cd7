/*
 * mela_gateway.h -- shared body of the six MEX gateways.
 *
 * Converts the mxArray arguments to mela_host_matrix, lets the library run
 * the reference gateway's checks and computation (mela_gateway), creates
 * the outputs through the MEX API and raises errors with the reference's
 * identifiers and messages.
 */
#ifndef MELA_GATEWAY_H
#define MELA_GATEWAY_H

#include "mex.h"
#include "mela.h"

typedef struct {
    mxArray **plhs;
} mela_mex_ctx;

static void *mela_mex_alloc(void *c, int32_t index, int32_t kind, int64_t rows, int64_t cols)
{
    mela_mex_ctx *x = (mela_mex_ctx *)c;
    mxArray *a;
    if (kind == MELA_KIND_DOUBLE && rows == 1 && cols == 1)
        a = mxCreateDoubleScalar(0.0);
    else if (kind == MELA_KIND_DOUBLE)
        a = mxCreateDoubleMatrix((mwSize)rows, (mwSize)cols, mxREAL);
    else
        a = mxCreateLogicalMatrix((mwSize)rows, (mwSize)cols);
    x->plhs[index] = a;
    return a ? mxGetData(a) : NULL;
}

static void mela_mex_run(int32_t fn, int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[])
{
    mela_host_matrix in[4];
    const mxArray *held[4] = {0, 0, 0, 0};
    int k = nrhs < 4 ? nrhs : 4;
    for (int i = 0; i < k; ++i) {
        const mxArray *a = prhs[i];
#ifdef MATLAB_MEX_FILE
        /* The rank gateways accept sparse input like the reference, but read
         * it through its full form instead of the sparse value array. */
        if (mxIsSparse(a) && (fn == MELA_FN_RANK_GF2 || fn == MELA_FN_RANK_M4RI)) {
            mxArray *full = NULL;
            mxArray *arg = (mxArray *)a;
            mexCallMATLAB(1, &full, 1, &arg, "full");
            held[i] = full;
            a = full;
        }
#endif
        in[i].kind = mxIsLogical(a) ? MELA_KIND_LOGICAL : (mxIsDouble(a) ? MELA_KIND_DOUBLE : MELA_KIND_OTHER);
        in[i].sparse = mxIsSparse(prhs[i]) ? 1 : 0;
        in[i].rows = (int64_t)mxGetM(a);
        in[i].cols = (int64_t)mxGetN(a);
        in[i].data = mxGetData(a);
    }
    (void)held;
    mela_mex_ctx c;
    c.plhs = plhs;
    mela_gateway_error e;
    if (mela_gateway(fn, nlhs, nrhs, in, mela_mex_alloc, &c, &e)) {
        if (e.id[0])
            mexErrMsgIdAndTxt(e.id, "%s", e.msg);
        else
            mexErrMsgTxt(e.msg);
    }
}

#endif /* MELA_GATEWAY_H */
