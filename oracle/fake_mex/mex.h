/* Minimal stand-in for MATLAB's mex.h (test infrastructure). */
#ifndef FAKE_MEX_MEX_H
#define FAKE_MEX_MEX_H
#include "matrix.h"
#ifdef __cplusplus
extern "C" {
#endif
/* Throws fake_mex::MexError (C++): the caller of mexFunction catches it. */
void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...);
#ifdef __cplusplus
}
#endif
#endif
