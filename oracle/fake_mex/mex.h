/* Minimal stand-in for MATLAB's mex.h (test infrastructure). */
#ifndef FAKE_MEX_MEX_H
#define FAKE_MEX_MEX_H
#include "matrix.h"
#ifdef __cplusplus
extern "C" {
#endif
/* Throws fake_mex::MexError (C++): the caller of mexFunction catches it. */
void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...);
/* Runs fn when the library is unloaded (here: never; kept for the API). */
int mexAtExit(void (*fn)(void));
/* The gateway every MEX file defines (C linkage, as in MATLAB's mex.h). */
void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]);
#ifdef __cplusplus
}
#endif
#endif
