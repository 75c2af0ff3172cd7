/* mela_null_m4ri -- MEX gateway (MATLAB name of the reference's src/mela_null_m4ri.c);
 * all checks and computation run in libmela_b200 (mela_gateway). */
#include "mela_gateway.h"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[])
{
    mela_mex_run(MELA_FN_NULL_M4RI, nlhs, plhs, nrhs, prhs);
}
