// Mixed-precision solver workspace and entry points (solve.cu, gemm_tc.cu).
#pragma once

#include "efie_internal.h"

struct SolveWork {
    int N = 0, ld = 0, nblk = 0;
    int epoch = 0;
    DevBuf planes;   // float re[N][ld], im[N][ld]  (row-major)
    DevBuf dinv;     // float2 [nblk][2][NB*NB]  (L^-1, U^-1 of each diagonal block)
    DevBuf vec;      // float2 rf[ld], y[ld], d[ld]
    DevBuf flags;    // int [2*nblk]
    DevBuf ctl;      // reductions, counters, flags (256 B)
    DevBuf packA, packB;  // tensor-core operand staging
};

int efie_solve_nb();
efie_status efie_mixed_workspace(SolveWork &w, int N);
efie_status efie_mixed_factor(efie_ctx *ctx, SolveWork &w, const void *Z);
efie_status efie_mixed_refine(efie_ctx *ctx, SolveWork &w, const void *Z, const void *b, void *x, double bnorm,
                              double tol, int max_iter, int *iters, double *relres, bool *converged);
efie_status efie_trsv(efie_ctx *ctx, SolveWork &w, bool lower, const float2 *rhs, float2 *out, void *x, int *flags,
                      int epoch, int *err, const int *skip);
efie_status efie_mixed_error_flag(efie_ctx *ctx, SolveWork &w, int *flag);
efie_status efie_port_reduce(efie_ctx *ctx, int N, const void *x, const double *wport, int model, int pe, int ge,
                             double V0, double Z0, void *out2);

// A22 -= L21 * U12 for the block at (k, kb): tensor cores when the trailing
// matrix is large enough, CUDA cores otherwise.
efie_status efie_trailing_update(efie_ctx *ctx, SolveWork &w, int k, int kb);
efie_status efie_trailing_update_simt(efie_ctx *ctx, SolveWork &w, int k, int kb);
extern "C" void efie_debug_disable_tensor_cores(int disable);
