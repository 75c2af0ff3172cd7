/*
 * matrix.h -- the subset of MATLAB's mxArray API that the mela_* MEX
 * gateways use, implemented by a small non-MATLAB host (mexhost.c).
 *
 * MATLAB itself is not needed to drive a MEX gateway: a gateway is a C
 * function `mexFunction(nlhs, plhs, nrhs, prhs)` over opaque mxArray
 * handles.  This host gives those handles a concrete layout (class, m x n,
 * column-major data) so the same gateway source can be compiled and called
 * from C or Python.  Function names and argument meanings follow MATLAB's
 * documented C Matrix API; only what the gateways call is provided.
 */
#ifndef MELA_MEXHOST_MATRIX_H
#define MELA_MEXHOST_MATRIX_H

#include <stddef.h>
#include <stdint.h>
#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef size_t mwSize;
typedef size_t mwIndex;
typedef bool mxLogical;

typedef enum {
    mxUNKNOWN_CLASS = 0,
    mxCELL_CLASS,
    mxSTRUCT_CLASS,
    mxLOGICAL_CLASS,
    mxCHAR_CLASS,
    mxVOID_CLASS,
    mxDOUBLE_CLASS,
    mxSINGLE_CLASS,
    mxINT8_CLASS,
    mxUINT8_CLASS,
    mxINT16_CLASS,
    mxUINT16_CLASS,
    mxINT32_CLASS,
    mxUINT32_CLASS,
    mxINT64_CLASS,
    mxUINT64_CLASS
} mxClassID;

/* Concrete layout of the host's arrays.  `data` is column-major, m*n
 * elements of the class's size.  `sparse` only flags the array (the host
 * keeps full storage): the gateways only ever ask mxIsSparse. */
typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;

typedef struct mxArray_tag {
    mxClassID classid;
    mwSize m, n;
    void *data;
    int sparse;
    int owns_data;
} mxArray;

mwSize mxGetM(const mxArray *a);
mwSize mxGetN(const mxArray *a);
bool mxIsDouble(const mxArray *a);
bool mxIsLogical(const mxArray *a);
bool mxIsSparse(const mxArray *a);
void *mxGetData(const mxArray *a);
double *mxGetPr(const mxArray *a);
mxLogical *mxGetLogicals(const mxArray *a);
mxClassID mxGetClassID(const mxArray *a);

mxArray *mxCreateLogicalMatrix(mwSize m, mwSize n);
mxArray *mxCreateDoubleScalar(double v);
mxArray *mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c);
void mxDestroyArray(mxArray *a);

void *mxCalloc(size_t n, size_t size);
void *mxMalloc(size_t n);
void mxFree(void *p);

#ifdef __cplusplus
}
#endif

#endif /* MELA_MEXHOST_MATRIX_H */
