/* [Z,Vrhs] = gassemble_ZV_EFIE_RWG_DIFF_GPU_FAST(V,F,E,plusTri,minusTri,plusSign,minusSign,
 *                                                rp,rm,Ap,Am,len,k,omega,mu,eps,exc)
 * Drop-in for gassemble_ZV_EFIE_RWG_DIFF_GPU_FAST.cu:125-435 over efie_gassemble_zv. */
#include "efie_mex_common.h"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    efie_mesh m;
    const double *excv;
    efie_c128 *Z, *V;
    efie_status s;
    efie_mex_check(nrhs == 17, "mex:args", "Expected 17 inputs.");
    efie_mex_check(nlhs == 2, "mex:args", "Expected 2 outputs [Z,Vrhs].");
    efie_mex_mesh(prhs, "mex:E", "E must be [Ne x 2] int32.", &m);
    efie_mex_check_rwg(prhs, (mwSize)m.Ne);
    efie_mex_check(mxIsDouble(prhs[16]) && mxGetNumberOfElements(prhs[16]) >= 5, "mex:exc",
                   "exc must be double vector len>=5: [patchEdge, groundEdge, V0, spreadRadius, selfAlpha].");
    excv = mxGetPr(prhs[16]);
    efie_mex_check((int)excv[0] >= 1 && (int)excv[0] <= m.Ne, "mex:port", "patchEdge out of range.");
    efie_mex_check((int)excv[1] >= 1 && (int)excv[1] <= m.Ne, "mex:port", "groundEdge out of range.");
    Z = (efie_c128 *)mxMalloc(sizeof(efie_c128) * (size_t)m.Ne * (size_t)m.Ne);
    V = (efie_c128 *)mxMalloc(sizeof(efie_c128) * (size_t)m.Ne);
    s = efie_gassemble_zv(efie_mex_ctx(), &m, efie_mex_cscalar(prhs[12]), mxGetScalar(prhs[13]),
                          mxGetScalar(prhs[14]), efie_mex_cscalar(prhs[15]), excv, Z, V);
    if (s != EFIE_OK) { mxFree(Z); mxFree(V); }
    efie_mex_status(s);
    plhs[0] = efie_mex_complex_out((mwSize)m.Ne, (mwSize)m.Ne, Z);
    plhs[1] = efie_mex_complex_out((mwSize)m.Ne, 1, V);
    mxFree(Z);
    mxFree(V);
}
