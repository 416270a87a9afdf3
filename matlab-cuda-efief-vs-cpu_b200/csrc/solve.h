// Mixed-precision solver, batched over frequencies (solve.cu, trsv.cu, gemm_tc.cu).
#pragma once

#include <cstdint>

#include "efie_internal.h"

constexpr int EFIE_MAX_BATCH = 64;

// Byte offset of element (row r, k) inside a K-major 64B-swizzled FP16 tile
// (the tensor-core operand layout): 16-byte chunk (k / 8) XOR (r / 2) mod 4,
// 8-row atoms of 512 bytes.
__host__ __device__ __forceinline__ uint32_t efie_swz64(uint32_t r, uint32_t k) {
    return r * 64u + ((((k >> 3) ^ (r >> 1)) & 3u) << 4) + ((k & 7u) << 1);
}

// The split's exact scale 2^(15-e) of a row (column) with largest magnitude
// mx: mx * 2^(15-e) in [2^14, 2^15), the top binade below FP16's largest
// power of two, so that the lo halves x - fp16(x) of entries down to 2^-18
// of the maximum are still normal FP16 numbers (with the maximum at 1/2..1
// they turn subnormal, and lose bits, below 2^-3); 1 for a zero maximum.  The
// exponent is capped so that the scale stays a finite FP32 power of two.
__device__ __forceinline__ float efie_pow2_scale(float mx) {
    if (!(mx > 0.f)) return 1.f;
    int e;
    frexpf(mx, &e);
    return ldexpf(1.f, min(15 - e, 126));
}

struct SolveWork {
    int N = 0, ld = 0, nblk = 0;
    int B = 0;                // batch slots (frequencies solved together)
    int epoch = 0;            // triangular-solve epoch (tags the progress counters)
    size_t pstride = 0;       // floats per frequency in `planes` (2 * ld * N)
    size_t dstride = 0;       // float2 per frequency in `dinv`
    int vstride = 0;          // float2 per frequency in each vector of `vec`
    int grid = 0;             // CTAs of the triangular-solve grid
    int kb_outer = 256;       // outer panel width of the two-level LU (K of the big updates)
    int tn_chain = 256;       // tile width (complex columns per CTA pair) of the K = 64 updates
    int tn_bulk = 256;        // ... and of the outer panels' updates
    bool resident_chain = false;   // K = 64 updates on resident, pipelined CTA pairs (k_update_tc_pipe)
    bool resident_bulk = false;    // the outer panels' updates likewise
    DevBuf planes;   // per f: float re[N][ld], im[N][ld]  (row-major)
    DevBuf dinv;     // per f: float2 [nblk][2][NB*NB] (L^-1, U^-1 of each diagonal block)
    DevBuf vec;      // float2 rf[B][vstride], y[B][vstride], d[B][vstride]
    DevBuf prog;     // triangular-solve progress counters: u64 [2][B][grid] on 64-byte lines
    DevBuf ctl;      // per f 64 bytes: red[3] @0, counter @24, conv @28, skip @32, err @36
    DevBuf rpart;    // residual-norm partial sums: double [B][ceil(N/32)]
    DevBuf active;   // int[B]: slot holds a frequency of this batch
    // int[B]: the slot whose complex64 factors (planes, dinv) precondition
    // slot f's refinement in a batch that shares the factors of an earlier
    // batch (the slot of the nearest factored frequency); read only while
    // fsrc_on, else every slot uses its own factors
    DevBuf fsrc;
    bool fsrc_on = false;
    // tensor-core operands, FP16 hi/lo packed once per panel (see PackView):
    // the outer panel's L and U by parity of the panel (packL[2], packU[2]),
    // the 64-wide block of the panel chain written by the panel kernel (ipL, ipU)
    DevBuf packL[2], packU[2], ipL, ipU;
    int ppitch = 0;       // packed rows (columns) per component plane
    // flexible GMRES (gmres.cu): Krylov basis V [M+1][B][N] and preconditioned
    // vectors Zm [M][B][N] in complex128, the new vector w [B][N], partial
    // sums and per-frequency Arnoldi state
    DevBuf gV, gZ, gw, gpart, gst, gflags;
    int gnch = 0;          // row chunks of the orthogonalisation kernels
    // Z is bit-exactly symmetric (symmetric gather): matrix-vector products read
    // only its upper triangle (128 x 128 tiles, partial vectors in spart)
    bool zsym = false;
    // with zsym, the complex64 LU is L D L^T from the lower part (about half
    // the trailing-update work); false: the general LU (the retry of a
    // frequency whose refinement missed its target)
    bool sym_lu = true;
    // the assembly writes the complex64 planes of each batch itself (symmetric
    // gather): the factorization starts without converting Z
    bool planes_from_assembly = false;
    DevBuf spart;
    // look-ahead LU: the panel chain runs on `hi` (highest priority) while the
    // bulk of each deferred trailing update runs on `lo`
    cudaStream_t hi = nullptr, lo = nullptr;
    cudaEvent_t ev_start = nullptr, ev_panel = nullptr, ev_rest = nullptr, ev_hi = nullptr;
    // max |Re|, |Im| of every row of each 64-column block of L (lmax[f][row][blk])
    // and of every column of each 64-row block of U (umax[f][blk][col]), written
    // with the factors; they give the split's power-of-two scales
    DevBuf lmax, umax;
    size_t mstride = 0;   // floats per frequency in lmax / umax (ld * nblk)
    // TMA tensor map (CUtensorMap) of the planes as float [B][2][N][ld], boxes
    // of 32 x 32: the tensor-core update adds its tiles into the factors with
    // bulk tensor reductions
    alignas(64) unsigned char planes_map[128] = {};
    // TMA tensor map of Z (complex128, all slots) for the GMRES products, and
    // the buffer, slot stride and sizes it was encoded for
    alignas(64) unsigned char zmap[128] = {};
    const void *zmap_base = nullptr;
    size_t zmap_stride = 0;
    int zmap_n = 0, zmap_b = 0;
    SolveWork() = default;
    SolveWork(const SolveWork &) = delete;
    SolveWork &operator=(const SolveWork &) = delete;
    ~SolveWork() {
        if (hi) cudaStreamDestroy(hi);
        if (lo) cudaStreamDestroy(lo);
        for (cudaEvent_t e : {ev_start, ev_panel, ev_rest, ev_hi})
            if (e) cudaEventDestroy(e);
    }
};

struct RefineResult {
    int iters = 0;
    double relres[EFIE_MAX_BATCH];
    bool converged[EFIE_MAX_BATCH];
    int err[EFIE_MAX_BATCH];
};

int efie_solve_nb();
efie_status efie_mixed_workspace(SolveWork &w, int N, int B, int kb_outer);
efie_status efie_mixed_factor(efie_ctx *ctx, SolveWork &w, const void *Z, size_t zstride, const int *active_host);
// The two halves of efie_mixed_factor: host-side set-up of a batch (control
// blocks, active mask), then the kernel sequence alone -- no allocation, no
// host copy, no synchronisation -- which plan_run captures once into a CUDA
// graph and replays for every batch.
efie_status efie_mixed_factor_prepare(efie_ctx *ctx, SolveWork &w, const int *active_host);
efie_status efie_mixed_factor_launch(efie_ctx *ctx, SolveWork &w, const void *Z, size_t zstride, int nact);
efie_status efie_gemm_workspace(SolveWork &w);
efie_status efie_mixed_refine(efie_ctx *ctx, SolveWork &w, const void *Z, size_t zstride, const void *b, void *x,
                              double bnorm, double tol, int max_iter, const int *active_host, RefineResult *res);
// Flexible GMRES on Z x = b with the complex64 LU as right preconditioner;
// the Arnoldi process and every vector are complex128.  Same contract as
// efie_mixed_refine (x starts at 0; res->iters counts matrix-vector products).
// x0_given: the active slots of x hold initial guesses (x = 0 otherwise).
efie_status efie_mixed_gmres(efie_ctx *ctx, SolveWork &w, const void *Z, size_t zstride, const void *b, void *x,
                             double bnorm, double tol, int max_iter, const int *active_host, RefineResult *res,
                             bool x0_given = false);
// r = b - Z x for every frequency of the batch (complex128), its complex64
// copy in w.vec, ||r|| / ||b|| and the convergence flags in w.ctl; r is also
// stored at rout + N f when rout is not null.
efie_status efie_true_residual(efie_ctx *ctx, SolveWork &w, const void *Z, size_t zstride, const void *x,
                               const void *b, double tol, void *rout, int nact);
// r = b - y for a precomputed y = Z x (complex128, [B][N]); otherwise as
// efie_true_residual.
efie_status efie_residual_finish(efie_ctx *ctx, SolveWork &w, const void *y, const void *b, double tol, void *rout,
                                 int nact);
// x = 0 for the active slots (the others keep theirs) and fresh control
// blocks (||b|| = bnorm) for every slot.
efie_status efie_refine_init(efie_ctx *ctx, SolveWork &w, void *x, double bnorm, bool zero_x = true);
// x_f = sum_t w[t][f] xs[idx[t][f]] over the terms t < 3 with idx >= 0, for
// the slots f < n (complex128 vectors of N).
struct GuessSpec {
    int idx[3][EFIE_MAX_BATCH];
    double w[3][EFIE_MAX_BATCH];
};
efie_status efie_interp_guess(efie_ctx *ctx, int N, int n, void *x, const void *xs, const GuessSpec &g);
efie_status efie_port_reduce(efie_ctx *ctx, int N, int B, const void *x, const double *wport, int model, int pe,
                             int ge, double V0, double Z0, void *out);

// Triangular solves of every active frequency in one cooperative launch.
efie_status efie_trsv_workspace(SolveWork &w);
efie_status efie_trsv(efie_ctx *ctx, SolveWork &w, bool lower, const float2 *rhs, float2 *out, void *x, int epoch);

// A view of packed tensor-core operands.  A panel of L (rows) or U (columns)
// is packed as half [B][nchunk][4][pitch][32]: per K chunk of 32 the
// components re hi, re lo, im hi, im lo (x = hi + lo after an exact
// power-of-two scaling of the row of L / column of U), each a plane of
// `pitch` rows of 32 K values in the 64-byte swizzle of the MMA operands, so
// that any 128 rows starting at a multiple of 8 are one contiguous 8 KB
// block.  The view's row 0 is row `off` of the packed panel.
struct PackView {
    const void *base = nullptr;   // __half, slot 0
    size_t stride = 0;            // halves per frequency slot
    int pitch = 0;
    int off = 0;
    PackView at(int o) const { PackView v = *this; v.off = off + o; return v; }
};
// Pack rows [r0, r1) of L over columns [kcol, kcol + K) (U: columns [c0, c1)
// over rows [krow, krow + K)) into `buf`; the view starts at r0 (c0).
efie_status efie_pack_l(efie_ctx *ctx, SolveWork &w, DevBuf &buf, int r0, int r1, int kcol, int K, PackView *out);
efie_status efie_pack_u(efie_ctx *ctx, SolveWork &w, DevBuf &buf, int c0, int c1, int krow, int K, PackView *out);
// The views of the 64-wide block packed by the panel kernel (rows / columns
// from s1 = k + 64 on).
PackView efie_inpanel_view(const SolveWork &w, bool lower);
// C[r0:r1, c0:c1] -= L[r0:r1, kcol:kcol+K] * U[krow:krow+K, c0:c1] for every
// active frequency: on the tensor cores from the packed views Lv (rows r0..)
// and Uv (columns c0..) when the block is large enough (K <= 256), else on
// CUDA cores from the factors (efie_update_simt, K <= 64 per call).
// tri_kb > 0 (a square block, r0 == c0): only the 256 x 256 tensor-core tiles
// that reach the block's lower triangle at tri_kb granularity (column block
// <= row block of width tri_kb, from r0), i.e. what a symmetric factorization
// with outer panels of tri_kb columns still reads.
efie_status efie_gemm_update(efie_ctx *ctx, SolveWork &w, int r0, int r1, int c0, int c1, int kcol, int krow, int K,
                             int nact, const PackView &Lv, const PackView &Uv, int tri_kb = 0);
// whether efie_gemm_update takes the tensor-core path for this block
bool efie_gemm_uses_tc(int rows, int cols, int K);
efie_status efie_update_simt(efie_ctx *ctx, SolveWork &w, int r0, int r1, int c0, int c1, int kcol, int krow, int K,
                             int nact);
extern "C" void efie_debug_disable_tensor_cores(int disable);
extern "C" void efie_debug_disable_symmetric_lu(int disable);
