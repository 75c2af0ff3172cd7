/* mela_rank_gf2 -- MEX gateway (MATLAB name of the reference's src/mela_rank_gf2.c);
 * all checks and computation run in libmela_b200 (mela_gateway). */
#include "mela_gateway.h"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[])
{
    mela_mex_run(MELA_FN_RANK_GF2, nlhs, plhs, nrhs, prhs);
}
