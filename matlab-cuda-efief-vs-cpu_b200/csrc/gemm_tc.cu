// Trailing-matrix update of the complex64 LU: A22 -= L21 * U12.
#include "solve.h"

efie_status efie_trailing_update(efie_ctx *ctx, SolveWork &w, int k, int kb, efie_sweep_stats *st, bool timing) {
    (void)st;
    (void)timing;
    return efie_trailing_update_simt(ctx, w, k, kb);
}
