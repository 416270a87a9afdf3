/* [Zin,S11] = patch_sweep_cuda(V,F,edge,plusTri,minusTri,plusSign,minusSign,rp,rm,Ap,Am,len,
 *                              freqs,mu,eps,patchEdge,groundEdge,V0,spreadRadius,Z0)
 * Drop-in for patch_sweep_cuda.cu:172-527 (centroid assembly, edge-difference
 * port) over efie_patch_sweep_centroid. */
#include "efie_mex_common.h"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    efie_mesh m;
    efie_c128 *Zin, *S11;
    mwSize Nf;
    int pe, ge;
    efie_status s;
    efie_mex_check(nrhs == 20, "mex:args", "Expected 20 inputs.");
    efie_mex_check(nlhs == 2, "mex:args", "Expected 2 outputs [Zin,S11].");
    efie_mex_mesh(prhs, "mex:edge", "edge must be [Ne x 2] int32.", &m);
    efie_mex_check_rwg(prhs, (mwSize)m.Ne);
    efie_mex_check(mxIsDouble(prhs[12]), "mex:freqs", "freqs must be double vector.");
    pe = (int)mxGetScalar(prhs[15]);
    ge = (int)mxGetScalar(prhs[16]);
    efie_mex_check(pe >= 1 && pe <= m.Ne, "mex:port", "patchEdge out of range.");
    efie_mex_check(ge >= 1 && ge <= m.Ne, "mex:port", "groundEdge out of range.");
    Nf = mxGetNumberOfElements(prhs[12]);
    Zin = (efie_c128 *)mxMalloc(sizeof(efie_c128) * (Nf ? Nf : 1));
    S11 = (efie_c128 *)mxMalloc(sizeof(efie_c128) * (Nf ? Nf : 1));
    s = efie_patch_sweep_centroid(efie_mex_ctx(), &m, mxGetPr(prhs[12]), (int32_t)Nf, mxGetScalar(prhs[13]),
                                  efie_mex_cscalar(prhs[14]), pe, ge, mxGetScalar(prhs[17]), mxGetScalar(prhs[18]),
                                  mxGetScalar(prhs[19]), NULL, Zin, S11, NULL, NULL);
    if (s != EFIE_OK) { mxFree(Zin); mxFree(S11); }
    efie_mex_status(s);
    plhs[0] = efie_mex_complex_out(Nf, 1, Zin);
    plhs[1] = efie_mex_complex_out(Nf, 1, S11);
    mxFree(Zin);
    mxFree(S11);
}
