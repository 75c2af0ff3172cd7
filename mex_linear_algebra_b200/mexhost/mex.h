/*
 * mex.h -- gateway-side MEX API of the non-MATLAB host (mexhost.c).
 *
 * mexErrMsgTxt / mexErrMsgIdAndTxt never return, as in MATLAB: they record
 * the message and long-jump back to mexhost_call(), which frees every block
 * the gateway obtained from mxCalloc/mxMalloc (MATLAB's memory manager does
 * the same on error).
 */
#ifndef MELA_MEXHOST_MEX_H
#define MELA_MEXHOST_MEX_H

#include "matrix.h"

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define MEXHOST_NORETURN __attribute__((noreturn))
#else
#define MEXHOST_NORETURN
#endif

void mexErrMsgTxt(const char *msg) MEXHOST_NORETURN;
void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...) MEXHOST_NORETURN;
int mexPrintf(const char *fmt, ...);

typedef void (*mexhost_gateway_fn)(int nlhs, mxArray *plhs[], int nrhs,
                                   const mxArray *prhs[]);

/* Call a gateway.  Returns 0 on success; on a mexErrMsg* error returns 1 and
 * copies the identifier (may be empty) and message into the caller buffers. */
int mexhost_call(mexhost_gateway_fn fn, int nlhs, mxArray *plhs[], int nrhs,
                 const mxArray *prhs[], char *err_id, size_t id_cap,
                 char *err_msg, size_t msg_cap);

/* Wrap caller-owned column-major storage as an mxArray (not freed by
 * mxDestroyArray). */
mxArray *mexhost_wrap(mxClassID cls, mwSize m, mwSize n, void *data, int sparse);

#ifdef __cplusplus
}
#endif

#endif /* MELA_MEXHOST_MEX_H */
