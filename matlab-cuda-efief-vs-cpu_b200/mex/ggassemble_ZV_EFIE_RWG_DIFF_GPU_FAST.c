/* [Z,Vrhs] = ggassemble_ZV_EFIE_RWG_DIFF_GPU_FAST(V,F,E,plusTri,minusTri,plusSign,minusSign,
 *                                                 rp,rm,Ap,Am,len,prepack,k,omega,mu,eps,excvec)
 * Drop-in for ggassemble_ZV_EFIE_RWG_DIFF_GPU_FAST.cu:542-843 over efie_ggassemble_zv. */
#include <stdlib.h>

#include "efie_mex_common.h"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    efie_mesh m;
    efie_prepack p;
    const double *excv;
    efie_c128 *Z, *V;
    efie_status s;
    efie_mex_check(nrhs == 18, "mex:args",
                   "Expected 18 inputs: V,F,E,plusTri,minusTri,plusSign,minusSign,rp,rm,Ap,Am,len,prepack,k,omega,mu,eps,excvec");
    efie_mex_check(nlhs == 2, "mex:args", "Expected 2 outputs [Z,Vrhs].");
    efie_mex_mesh(prhs, "mex:E", "E must be [Ne x 2] int32.", &m);
    efie_mex_check(mxIsStruct(prhs[12]), "mex:prepack", "prepack must be a struct from efie_precompute_pack.");
    efie_mex_check(mxIsDouble(prhs[17]) && mxGetNumberOfElements(prhs[17]) >= 4, "mex:exc",
                   "excvec must be [patchEdge, groundEdge, V0, spreadRadius].");
    excv = mxGetPr(prhs[17]);
    efie_mex_check((int)excv[0] >= 1 && (int)excv[0] <= m.Ne, "mex:port", "patchEdge out of range.");
    efie_mex_check((int)excv[1] >= 1 && (int)excv[1] <= m.Ne, "mex:port", "groundEdge out of range.");
    efie_mex_prepack(prhs[12], "self_a", 1, (mwSize)m.Nt, &p);
    Z = (efie_c128 *)mxMalloc(sizeof(efie_c128) * (size_t)m.Ne * (size_t)m.Ne);
    V = (efie_c128 *)mxMalloc(sizeof(efie_c128) * (size_t)m.Ne);
    s = efie_ggassemble_zv(efie_mex_ctx(), &m, &p, efie_mex_cscalar(prhs[13]), mxGetScalar(prhs[14]),
                           mxGetScalar(prhs[15]), efie_mex_cscalar(prhs[16]), excv, Z, V);
    if (s != EFIE_OK) { mxFree(Z); mxFree(V); }
    efie_mex_status(s);
    plhs[0] = efie_mex_complex_out((mwSize)m.Ne, (mwSize)m.Ne, Z);
    plhs[1] = efie_mex_complex_out((mwSize)m.Ne, 1, V);
    mxFree(Z);
    mxFree(V);
}
