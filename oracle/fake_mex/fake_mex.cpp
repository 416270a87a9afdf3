// Implementation of the fake mex/matrix API plus a small C driver so that a
// test harness (ctypes) can build mxArrays, call mexFunction and read the
// outputs.  Test infrastructure only.
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "mex.h"

struct mxArray_tag {
    mxClassID cls = mxUNKNOWN_CLASS;
    std::vector<mwSize> dims;
    void *pr = nullptr;
    void *pi = nullptr;
    std::vector<std::string> names;
    std::vector<mxArray *> fields;
};

namespace fake_mex {
struct MexError : std::runtime_error {
    std::string id;
    MexError(const char *i, const std::string &m) : std::runtime_error(m), id(i) {}
};
static size_t elsize(mxClassID c) {
    switch (c) {
    case mxDOUBLE_CLASS: return 8;
    case mxINT32_CLASS: return 4;
    case mxUINT8_CLASS: return 1;
    default: return 0;
    }
}
}  // namespace fake_mex

extern "C" {
mwSize mxGetNumberOfElements(const mxArray *a) {
    mwSize n = 1;
    for (mwSize d : a->dims) n *= d;
    return n;
}
mwSize mxGetM(const mxArray *a) { return a->dims.empty() ? 0 : a->dims[0]; }
mwSize mxGetN(const mxArray *a) {
    mwSize n = 1;
    for (size_t i = 1; i < a->dims.size(); i++) n *= a->dims[i];
    return n;
}
mwSize mxGetNumberOfDimensions(const mxArray *a) { return a->dims.size(); }
const mwSize *mxGetDimensions(const mxArray *a) { return a->dims.data(); }
int mxIsDouble(const mxArray *a) { return a->cls == mxDOUBLE_CLASS; }
int mxIsInt32(const mxArray *a) { return a->cls == mxINT32_CLASS; }
int mxIsUint8(const mxArray *a) { return a->cls == mxUINT8_CLASS; }
int mxIsStruct(const mxArray *a) { return a->cls == mxSTRUCT_CLASS; }
int mxIsComplex(const mxArray *a) { return a->pi != nullptr; }
double mxGetScalar(const mxArray *a) {
    if (!a->pr || mxGetNumberOfElements(a) == 0) return 0.0;
    switch (a->cls) {
    case mxDOUBLE_CLASS: return ((double *)a->pr)[0];
    case mxINT32_CLASS: return ((int32_t *)a->pr)[0];
    case mxUINT8_CLASS: return ((uint8_t *)a->pr)[0];
    default: return 0.0;
    }
}
double *mxGetPr(const mxArray *a) { return (double *)a->pr; }
double *mxGetPi(const mxArray *a) { return (double *)a->pi; }
double *mxGetDoubles(const mxArray *a) { return (double *)a->pr; }
mxComplexDouble *mxGetComplexDoubles(const mxArray *) { return nullptr; }
void *mxGetData(const mxArray *a) { return a->pr; }
mxArray *mxGetField(const mxArray *a, mwIndex, const char *name) {
    for (size_t i = 0; i < a->names.size(); i++)
        if (a->names[i] == name) return a->fields[i];
    return nullptr;
}
mxArray *mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c) {
    mxArray *a = new mxArray_tag();
    a->cls = mxDOUBLE_CLASS;
    a->dims = {m, n};
    a->pr = calloc(m * n ? m * n : 1, 8);
    if (c == mxCOMPLEX) a->pi = calloc(m * n ? m * n : 1, 8);
    return a;
}
void *mxMalloc(size_t n) { return malloc(n ? n : 1); }
void mxFree(void *p) { free(p); }
void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    throw fake_mex::MexError(id, buf);
}

// ---- driver API ----
mxArray *fm_numeric(int cls, int ndims, const size_t *dims, const void *re, const void *im) {
    mxArray *a = new mxArray_tag();
    a->cls = (mxClassID)cls;
    a->dims.assign(dims, dims + ndims);
    size_t n = mxGetNumberOfElements(a) * fake_mex::elsize(a->cls);
    a->pr = calloc(n ? n : 1, 1);
    if (re && n) memcpy(a->pr, re, n);
    if (im) {
        a->pi = calloc(n ? n : 1, 1);
        if (n) memcpy(a->pi, im, n);
    }
    return a;
}
mxArray *fm_struct(int nf, const char **names, mxArray **vals) {
    mxArray *a = new mxArray_tag();
    a->cls = mxSTRUCT_CLASS;
    a->dims = {1, 1};
    for (int i = 0; i < nf; i++) {
        a->names.push_back(names[i]);
        a->fields.push_back(vals[i]);
    }
    return a;
}
void fm_destroy(mxArray *a) {
    if (!a) return;
    for (mxArray *f : a->fields) fm_destroy(f);
    free(a->pr);
    free(a->pi);
    delete a;
}
size_t fm_numel(const mxArray *a) { return mxGetNumberOfElements(a); }
void fm_read(const mxArray *a, double *re, double *im) {
    size_t n = mxGetNumberOfElements(a);
    if (re) memcpy(re, a->pr, n * 8);
    if (im) {
        if (a->pi) memcpy(im, a->pi, n * 8);
        else memset(im, 0, n * 8);
    }
}
}

int mexAtExit(void (*)(void)) { return 0; }

// Calls mexFunction; returns 0 on success, 1 with the error id/message copied out.
extern "C" int fm_call(int nlhs, mxArray **plhs, int nrhs, const mxArray **prhs, char *id, char *msg, int cap) {
    try {
        mexFunction(nlhs, plhs, nrhs, prhs);
        return 0;
    } catch (const fake_mex::MexError &e) {
        snprintf(id, cap, "%s", e.id.c_str());
        snprintf(msg, cap, "%s", e.what());
        return 1;
    }
}
