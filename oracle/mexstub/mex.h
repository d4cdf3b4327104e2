/* LINK-CHECK STUB -- not MATLAB's header (see matrix.h beside it).
 * Declares the documented MEX entry points the reference's gateway calls. */
#ifndef SPEIGS_MEXSTUB_MEX_H
#define SPEIGS_MEXSTUB_MEX_H
#include "matrix.h"

void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...);
void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]);
#endif
