/* Minimal stand-in for MATLAB's matrix.h (separate-complex API, -R2017b
 * layout).  Test infrastructure: lets MEX sources compile and run without
 * MATLAB.  Only the subset used by the EFIE MEX files is provided. */
#ifndef FAKE_MEX_MATRIX_H
#define FAKE_MEX_MATRIX_H
#include <stddef.h>
#include <stdint.h>

#ifndef MX_HAS_INTERLEAVED_COMPLEX
#define MX_HAS_INTERLEAVED_COMPLEX 0
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef size_t mwSize;
typedef size_t mwIndex;
typedef struct mxArray_tag mxArray;
typedef enum { mxUNKNOWN_CLASS = 0, mxSTRUCT_CLASS = 2, mxDOUBLE_CLASS = 6, mxINT32_CLASS = 12,
               mxUINT8_CLASS = 9 } mxClassID;
typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;
typedef struct { double real, imag; } mxComplexDouble;

mwSize mxGetM(const mxArray *a);
mwSize mxGetN(const mxArray *a);
mwSize mxGetNumberOfElements(const mxArray *a);
mwSize mxGetNumberOfDimensions(const mxArray *a);
const mwSize *mxGetDimensions(const mxArray *a);
int mxIsDouble(const mxArray *a);
int mxIsInt32(const mxArray *a);
int mxIsUint8(const mxArray *a);
int mxIsStruct(const mxArray *a);
int mxIsComplex(const mxArray *a);
double mxGetScalar(const mxArray *a);
double *mxGetPr(const mxArray *a);
double *mxGetPi(const mxArray *a);
double *mxGetDoubles(const mxArray *a);
mxComplexDouble *mxGetComplexDoubles(const mxArray *a);
void *mxGetData(const mxArray *a);
mxArray *mxGetField(const mxArray *a, mwIndex i, const char *name);
mxArray *mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c);
void *mxMalloc(size_t n);
void mxFree(void *p);

#ifdef __cplusplus
}
#endif
#endif
