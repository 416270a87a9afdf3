/* Shared marshalling for the MEX wrappers over libefie_b200 (include/efie_b200.h).
 * Build with MATLAB:   mex -R2017b -I<repo>/include <file>.c -L<repo>/matlab-cuda-efief-vs-cpu_b200 -lefie_b200
 * Every wrapper keeps the reference's signature, argument checks and error
 * identifiers; computation happens behind the C ABI. */
#ifndef EFIE_MEX_COMMON_H
#define EFIE_MEX_COMMON_H
#include <string.h>

#include "efie_b200.h"
#include "mex.h"

static efie_ctx *g_efie_ctx = NULL;

static inline void efie_mex_release(void) {
    if (g_efie_ctx) efie_ctx_destroy(g_efie_ctx);
    g_efie_ctx = NULL;
}

static inline void efie_mex_check(int cond, const char *id, const char *msg) {
    if (!cond) mexErrMsgIdAndTxt(id, msg);
}

static inline void efie_mex_status(efie_status s) {
    if (s != EFIE_OK) mexErrMsgIdAndTxt(efie_status_id(s), "%s", efie_last_error());
}

/* One context per MATLAB session, released by mexAtExit. */
static inline efie_ctx *efie_mex_ctx(void) {
    if (!g_efie_ctx) {
        efie_mex_status(efie_ctx_create(0, &g_efie_ctx));
        mexAtExit(efie_mex_release);
    }
    return g_efie_ctx;
}

static inline efie_c128 efie_mex_cscalar(const mxArray *a) {
    efie_c128 z;
    z.re = mxGetScalar(a);
    z.im = 0.0;
    if (mxIsComplex(a)) {
#if MX_HAS_INTERLEAVED_COMPLEX
        z.im = mxGetComplexDoubles(a)[0].imag;
#else
        if (mxGetPi(a)) z.im = mxGetPi(a)[0];
#endif
    }
    return z;
}

/* V,F,E,plusTri,minusTri,plusSign,minusSign,rp,rm,Ap,Am,len = prhs[0..11] */
static inline void efie_mex_mesh(const mxArray *prhs[], const char *e_id, const char *e_msg, efie_mesh *m) {
    efie_mex_check(mxIsDouble(prhs[0]) && mxGetN(prhs[0]) == 3, "mex:V", "V must be [Nv x 3] double.");
    efie_mex_check(mxIsInt32(prhs[1]) && mxGetN(prhs[1]) == 3, "mex:F", "F must be [Nt x 3] int32.");
    efie_mex_check(mxIsInt32(prhs[2]) && mxGetN(prhs[2]) == 2, e_id, e_msg);
    m->Nv = (int32_t)mxGetM(prhs[0]);
    m->Nt = (int32_t)mxGetM(prhs[1]);
    m->Ne = (int32_t)mxGetM(prhs[2]);
    m->V = mxGetPr(prhs[0]);
    m->F = (const int32_t *)mxGetData(prhs[1]);
    m->E = (const int32_t *)mxGetData(prhs[2]);
    m->plusTri = (const int32_t *)mxGetData(prhs[3]);
    m->minusTri = (const int32_t *)mxGetData(prhs[4]);
    m->plusSign = (const int32_t *)mxGetData(prhs[5]);
    m->minusSign = (const int32_t *)mxGetData(prhs[6]);
    m->rp = mxGetPr(prhs[7]);
    m->rm = mxGetPr(prhs[8]);
    m->Ap = mxGetPr(prhs[9]);
    m->Am = mxGetPr(prhs[10]);
    m->len = mxGetPr(prhs[11]);
}

/* gassemble_ZV_EFIE_RWG_DIFF_GPU_FAST.cu:181-191 / patch_sweep_cuda.cu:210-219 */
static inline void efie_mex_check_rwg(const mxArray *prhs[], mwSize Ne) {
    static const char *names[4] = {"plusTri", "minusTri", "plusSign", "minusSign"};
    static const char *ids[4] = {"mex:plusTri", "mex:minusTri", "mex:plusSign", "mex:minusSign"};
    static const char *msgs[4] = {"plusTri must be int32 [Ne x 1].", "minusTri must be int32 [Ne x 1].",
                                  "plusSign must be int32 [Ne x 1].", "minusSign must be int32 [Ne x 1]."};
    int i;
    (void)names;
    for (i = 0; i < 4; i++) efie_mex_check(mxIsInt32(prhs[3 + i]) && mxGetM(prhs[3 + i]) == Ne, ids[i], msgs[i]);
    efie_mex_check(mxIsDouble(prhs[7]) && mxGetM(prhs[7]) == Ne && mxGetN(prhs[7]) == 3, "mex:rp", "rp must be [Ne x 3] double.");
    efie_mex_check(mxIsDouble(prhs[8]) && mxGetM(prhs[8]) == Ne && mxGetN(prhs[8]) == 3, "mex:rm", "rm must be [Ne x 3] double.");
    efie_mex_check(mxIsDouble(prhs[9]) && mxGetNumberOfElements(prhs[9]) == Ne, "mex:Ap", "Ap must be [Ne x 1] double.");
    efie_mex_check(mxIsDouble(prhs[10]) && mxGetNumberOfElements(prhs[10]) == Ne, "mex:Am", "Am must be [Ne x 1] double.");
    efie_mex_check(mxIsDouble(prhs[11]) && mxGetNumberOfElements(prhs[11]) == Ne, "mex:len", "len must be [Ne x 1] double.");
}

static inline const mxArray *efie_mex_field(const mxArray *s, const char *name, const char *id, const char *msg) {
    const mxArray *f = mxGetField(s, 0, name);
    efie_mex_check(f != NULL, id, msg);
    return f;
}

/* prepack struct of efie_precompute_pack.m:43-58 (dimensions as fastquad.cu:559-567) */
static inline void efie_mex_prepack(const mxArray *pre, const char *self_a_name, int check_dims, mwSize Nt,
                             efie_prepack *p) {
    const mxArray *r_reg = efie_mex_field(pre, "r_reg", "mex:prepack", "Missing field in prepack.");
    const mxArray *w_reg = efie_mex_field(pre, "w_reg", "mex:prepack", "Missing field in prepack.");
    const mxArray *nearMat = efie_mex_field(pre, "nearMat", "mex:prepack", "Missing field in prepack.");
    const mxArray *self_r = efie_mex_field(pre, "self_r", "mex:prepack", "Missing field in prepack.");
    const mxArray *self_w = efie_mex_field(pre, "self_w", "mex:prepack", "Missing field in prepack.");
    const mxArray *self_a = efie_mex_field(pre, self_a_name, "mex:prepack", "Missing field in prepack.");
    const mxArray *near_r = efie_mex_field(pre, "near_r", "mex:prepack", "Missing field in prepack.");
    const mxArray *near_w = efie_mex_field(pre, "near_w", "mex:prepack", "Missing field in prepack.");
    const mxArray *aeqTri = efie_mex_field(pre, "aeqTri", "mex:prepack", "Missing field in prepack.");
    const mxArray *near_alpha = efie_mex_field(pre, "near_alpha", "mex:prepack", "Missing field in prepack.");
    const mwSize *dr, *ds, *dn;
    if (check_dims) { /* ggassemble_ZV_EFIE_RWG_DIFF_GPU_FAST.cu:629-657 */
        efie_mex_check(mxIsDouble(r_reg) && mxGetNumberOfDimensions(r_reg) == 3, "mex:r_reg", "r_reg must be [Nq x 3 x Nt] double.");
        efie_mex_check(mxIsDouble(w_reg) && mxGetNumberOfDimensions(w_reg) == 2, "mex:w_reg", "w_reg must be [Nq x Nt] double.");
        efie_mex_check(mxIsUint8(nearMat), "mex:nearMat", "nearMat must be uint8 [Nt x Nt].");
        efie_mex_check(mxIsDouble(self_r) && mxGetNumberOfDimensions(self_r) == 4, "mex:self_r", "self_r must be [Nq2 x 3 x NsS x Nt].");
        efie_mex_check(mxIsDouble(self_w) && mxGetNumberOfDimensions(self_w) == 3, "mex:self_w", "self_w must be [Nq2 x NsS x Nt].");
        efie_mex_check(mxIsDouble(self_a) && mxGetNumberOfDimensions(self_a) == 2, "mex:self_a", "self_a must be [NsS x Nt].");
        efie_mex_check(mxIsDouble(near_r) && mxGetNumberOfDimensions(near_r) == 4, "mex:near_r", "near_r must be [Nq2 x 3 x NsN x Nt].");
        efie_mex_check(mxIsDouble(near_w) && mxGetNumberOfDimensions(near_w) == 3, "mex:near_w", "near_w must be [Nq2 x NsN x Nt].");
        efie_mex_check(mxIsDouble(aeqTri) && mxGetNumberOfElements(aeqTri) == Nt, "mex:aeqTri", "aeqTri must be [Nt x 1].");
        dr = mxGetDimensions(r_reg);
        efie_mex_check(dr[1] == 3, "mex:r_reg", "r_reg dim2 must be 3.");
        efie_mex_check(dr[2] == Nt, "mex:r_reg", "r_reg dim3 must be Nt.");
        ds = mxGetDimensions(self_r);
        efie_mex_check(ds[1] == 3, "mex:self_r", "self_r dim2 must be 3.");
        efie_mex_check(ds[3] == Nt, "mex:self_r", "self_r dim4 must be Nt.");
        dn = mxGetDimensions(near_r);
        efie_mex_check(dn[0] == ds[0], "mex:near_r", "near_r Nq2 mismatch.");
        efie_mex_check(dn[3] == Nt, "mex:near_r", "near_r dim4 must be Nt.");
    }
    efie_mex_check(mxGetNumberOfDimensions(self_r) >= 3 && mxGetNumberOfDimensions(near_r) >= 3, "mex:prepack",
                   "prepack must be a struct from efie_precompute_pack.");
    dr = mxGetDimensions(r_reg);
    ds = mxGetDimensions(self_r);
    dn = mxGetDimensions(near_r);
    p->Nt = (int32_t)Nt;
    p->Nq = (int32_t)dr[0];
    p->Nq2 = (int32_t)ds[0];
    p->NsS = (int32_t)ds[2];
    p->NsN = (int32_t)dn[2];
    p->r_reg = mxGetPr(r_reg);
    p->w_reg = mxGetPr(w_reg);
    p->nearMat = (uint8_t *)mxGetData(nearMat);
    p->self_r = mxGetPr(self_r);
    p->self_w = mxGetPr(self_w);
    p->self_a = mxGetPr(self_a);
    p->near_r = mxGetPr(near_r);
    p->near_w = mxGetPr(near_w);
    p->aeqTri = mxGetPr(aeqTri);
    p->near_alpha = mxGetScalar(near_alpha);
    p->self_alpha = 0.0;
}

/* Complex [m x n] output from interleaved complex128 data. */
static inline mxArray *efie_mex_complex_out(mwSize m, mwSize n, const efie_c128 *src) {
    mxArray *a = mxCreateDoubleMatrix(m, n, mxCOMPLEX);
    mwSize i, N = m * n;
#if MX_HAS_INTERLEAVED_COMPLEX
    mxComplexDouble *z = mxGetComplexDoubles(a);
    for (i = 0; i < N; i++) { z[i].real = src[i].re; z[i].imag = src[i].im; }
#else
    double *re = mxGetPr(a), *im = mxGetPi(a);
    for (i = 0; i < N; i++) { re[i] = src[i].re; im[i] = src[i].im; }
#endif
    return a;
}
#endif
