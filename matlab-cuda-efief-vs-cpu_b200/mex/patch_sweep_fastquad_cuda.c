/* [Zin,S11] = patch_sweep_fastquad_cuda(V,F,E,plusTri,minusTri,plusSign,minusSign,rp,rm,Ap,Am,len,
 *                                       prepack,freqs,mu,eps,patchEdge,groundEdge,V0,spreadRadius,Z0)
 * Drop-in for patch_sweep_fastquad_cuda.cu:461-844 over efie_patch_sweep_fastquad
 * (mixed-precision solver with FP64 refinement to 1e-10; set EFIE_SOLVER=fp64 in
 * the environment for the complex128 LU). */
#include <stdlib.h>
#include <string.h>

#include "efie_mex_common.h"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    efie_mesh m;
    efie_prepack p;
    efie_sweep_opts o;
    efie_c128 *Zin, *S11;
    mwSize Nf;
    int pe, ge;
    const char *solver;
    efie_status s;
    efie_mex_check(nrhs == 21, "mex:args", "Expected 21 inputs.");
    efie_mex_check(nlhs == 2, "mex:args", "Expected 2 outputs [Zin,S11].");
    efie_mex_mesh(prhs, "mex:E", "E must be [Ne x 2] int32.", &m);
    efie_mex_check(mxIsDouble(prhs[13]), "mex:freqs", "freqs must be double vector.");
    efie_mex_check(mxIsStruct(prhs[12]), "mex:prepack", "prepack must be struct.");
    pe = (int)mxGetScalar(prhs[16]);
    ge = (int)mxGetScalar(prhs[17]);
    efie_mex_check(pe >= 1 && pe <= m.Ne, "mex:port", "patchEdge out of range.");
    efie_mex_check(ge >= 1 && ge <= m.Ne, "mex:port", "groundEdge out of range.");
    efie_mex_prepack(prhs[12], "self_a", 0, (mwSize)m.Nt, &p);
    Nf = mxGetNumberOfElements(prhs[13]);
    efie_sweep_opts_default(&o);
    solver = getenv("EFIE_SOLVER");
    if (solver && strcmp(solver, "fp64") == 0) o.solver = EFIE_SOLVER_FP64;
    Zin = (efie_c128 *)mxMalloc(sizeof(efie_c128) * (Nf ? Nf : 1));
    S11 = (efie_c128 *)mxMalloc(sizeof(efie_c128) * (Nf ? Nf : 1));
    s = efie_patch_sweep_fastquad(efie_mex_ctx(), &m, &p, mxGetPr(prhs[13]), (int32_t)Nf, mxGetScalar(prhs[14]),
                                  efie_mex_cscalar(prhs[15]), pe, ge, mxGetScalar(prhs[18]), mxGetScalar(prhs[19]),
                                  mxGetScalar(prhs[20]), &o, Zin, S11, NULL, NULL);
    if (s != EFIE_OK) { mxFree(Zin); mxFree(S11); }
    efie_mex_status(s);
    plhs[0] = efie_mex_complex_out(Nf, 1, Zin);
    plhs[1] = efie_mex_complex_out(Nf, 1, S11);
    mxFree(Zin);
    mxFree(S11);
}
