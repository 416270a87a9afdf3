/*
 * efie_b200.h -- C ABI of the B200-native EFIE method-of-moments hot path.
 *
 * Drop-in boundary for the reference's CUDA MEX entry points
 * (mahmut26/Matlab-cuda-efief-vs-cpu).  Every entry point takes plain host
 * pointers laid out exactly as MATLAB hands them to a MEX function:
 * column-major arrays, 1-based int32 index values, complex128 as interleaved
 * (re, im) pairs.  No torch or CUDA types appear in the signatures.  A MEX
 * wrapper only marshals mxArray <-> pointers and maps efie_status to the
 * reference's error identifiers with efie_status_id().
 *
 * Threading: a context is not thread-safe; use one context per host thread.
 * Errors never leak device memory: buffers are owned by the context (or plan)
 * and released by efie_ctx_destroy / efie_plan_destroy.
 */
#ifndef EFIE_B200_H
#define EFIE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { double re, im; } efie_c128;

/* Status codes.  efie_status_id() returns the reference's mexErrMsgIdAndTxt
 * identifier for each (e.g. "mex:port"); the message of the last failure on
 * the calling thread is returned by efie_last_error(). */
typedef enum efie_status {
    EFIE_OK = 0,
    EFIE_ERR_ARGS = 1,        /* mex:args     */
    EFIE_ERR_V = 2,           /* mex:V        */
    EFIE_ERR_F = 3,           /* mex:F        */
    EFIE_ERR_E = 4,           /* mex:E        */
    EFIE_ERR_RWG = 5,         /* mex:rwg  (plusTri/minusTri/sign/rp/rm/Ap/Am/len) */
    EFIE_ERR_PORT = 6,        /* mex:port     */
    EFIE_ERR_PREPACK = 7,     /* mex:prepack  */
    EFIE_ERR_R_REG = 8,       /* mex:r_reg    */
    EFIE_ERR_W_REG = 9,       /* mex:w_reg    */
    EFIE_ERR_NEARMAT = 10,    /* mex:nearMat  */
    EFIE_ERR_SELF_R = 11,     /* mex:self_r   */
    EFIE_ERR_SELF_W = 12,     /* mex:self_w   */
    EFIE_ERR_SELF_A = 13,     /* mex:self_a   */
    EFIE_ERR_NEAR_R = 14,     /* mex:near_r   */
    EFIE_ERR_NEAR_W = 15,     /* mex:near_w   */
    EFIE_ERR_AEQTRI = 16,     /* mex:aeqTri   */
    EFIE_ERR_RHS = 17,        /* mex:rhs      */
    EFIE_ERR_EPS = 18,        /* mex:eps      */
    EFIE_ERR_EXC = 19,        /* mex:exc      */
    EFIE_ERR_FREQS = 20,      /* mex:freqs    */
    EFIE_ERR_CUDA = 21,       /* cuda:rt      */
    EFIE_ERR_CUSOLVER = 22,   /* cuda:cusolver */
    EFIE_ERR_SINGULAR = 23,   /* efie:singular  (LU pivot zero; the reference never checks info) */
    EFIE_ERR_NOMEM = 24,      /* efie:nomem     */
    EFIE_ERR_TIMEOUT = 25,    /* efie:timeout   (a bounded device wait gave up) */
    EFIE_ERR_MESH = 26        /* efie:mesh      (topology error in the mesh builders) */
} efie_status;

const char *efie_status_id(efie_status s);
const char *efie_last_error(void);

/* ---------------------------------------------------------------------- */
/* Context                                                                 */
/* ---------------------------------------------------------------------- */
typedef struct efie_ctx efie_ctx;

efie_status efie_ctx_create(int device, efie_ctx **out);
void efie_ctx_destroy(efie_ctx *ctx);
/* Launch every kernel of this context on `stream` (a cudaStream_t, 0 = the
 * context's own stream). */
efie_status efie_ctx_set_stream(efie_ctx *ctx, void *stream);

/* ---------------------------------------------------------------------- */
/* Boundary data: the arrays the MEX entry points receive                  */
/* ---------------------------------------------------------------------- */

/* V,F,E,plusTri,minusTri,plusSign,minusSign,rp,rm,Ap,Am,len
 * (patch_sweep_fastquad_cuda.cu:463-471; ggassemble_ZV_EFIE_RWG_DIFF_GPU_FAST.cu:548-559) */
typedef struct efie_mesh {
    int32_t Nv, Nt, Ne;
    const double *V;           /* [Nv x 3]                           */
    const int32_t *F;          /* [Nt x 3] 1-based                   */
    const int32_t *E;          /* [Ne x 2] 1-based  (rwg.edge)       */
    const int32_t *plusTri;    /* [Ne] 1-based                       */
    const int32_t *minusTri;   /* [Ne] 1-based                       */
    const int32_t *plusSign;   /* [Ne] +1/-1                         */
    const int32_t *minusSign;  /* [Ne] +1/-1                         */
    const double *rp, *rm;     /* [Ne x 3] free vertices             */
    const double *Ap, *Am;     /* [Ne] triangle areas                */
    const double *len;         /* [Ne] edge lengths                  */
} efie_mesh;

/* The prepack struct of efie_precompute_pack.m:43-58 (dimensions as read by
 * patch_sweep_fastquad_cuda.cu:559-567).  Pointers are read-only inputs for
 * the assembly entry points and outputs of efie_precompute_pack(). */
typedef struct efie_prepack {
    int32_t Nt, Nq, Nq2, NsS, NsN;
    double *r_reg;             /* [Nq x 3 x Nt]                      */
    double *w_reg;             /* [Nq x Nt]   (weights include 2A)   */
    uint8_t *nearMat;          /* [Nt x Nt]                          */
    double *self_r;            /* [Nq2 x 3 x NsS x Nt]               */
    double *self_w;            /* [Nq2 x NsS x Nt]                   */
    double *self_a;            /* [NsS x Nt]                         */
    double *near_r;            /* [Nq2 x 3 x NsN x Nt]               */
    double *near_w;            /* [Nq2 x NsN x Nt]                   */
    double *aeqTri;            /* [Nt]                               */
    double near_alpha;
    double self_alpha;         /* carried, unused by the kernels (as in the reference) */
} efie_prepack;

/* ---------------------------------------------------------------------- */
/* Assembly-only entry points                                              */
/* ---------------------------------------------------------------------- */

/* Replaces ggassemble_ZV_EFIE_RWG_DIFF_GPU_FAST.cu:542-843 (mexFunction):
 * [Z,Vrhs] = ggassemble_...(V,F,E,plusTri,minusTri,plusSign,minusSign,rp,rm,
 *                            Ap,Am,len,prepack,k,omega,mu,eps,excvec)
 * excvec = [patchEdge, groundEdge, V0, spreadRadius].
 * Z: [Ne x Ne] complex128 column-major; Vrhs: [Ne] complex128 (imag 0). */
efie_status efie_ggassemble_zv(efie_ctx *ctx, const efie_mesh *mesh, const efie_prepack *pre,
                               efie_c128 k, double omega, double mu, efie_c128 eps,
                               const double excvec[4], efie_c128 *Z, efie_c128 *Vrhs);

/* Replaces gassemble_ZV_EFIE_RWG_DIFF_GPU_FAST.cu:125-435 (mexFunction), the
 * one-point centroid assembly: exc = [patchEdge, groundEdge, V0,
 * spreadRadius, selfAlpha]. */
efie_status efie_gassemble_zv(efie_ctx *ctx, const efie_mesh *mesh,
                              efie_c128 k, double omega, double mu, efie_c128 eps,
                              const double exc[5], efie_c128 *Z, efie_c128 *Vrhs);

/* ---------------------------------------------------------------------- */
/* Frequency sweeps (assemble + solve + port reduction per frequency)      */
/* ---------------------------------------------------------------------- */
typedef enum efie_solver {
    EFIE_SOLVER_FP64 = 0,   /* complex128 LU (cuSOLVER Zgetrf/Zgetrs), the plain FP64 GPU path */
    EFIE_SOLVER_MIXED = 1   /* complex64 tensor-core LU + FP64 iterative refinement           */
} efie_solver;

typedef enum efie_port_model {
    EFIE_PORT_GAUSS = 0,     /* Iport = sum((wPatch - wGnd) .* len .* I)  (fastquad.cu:777-785) */
    EFIE_PORT_EDGE_DIFF = 1  /* Iport = I(patchEdge) - I(groundEdge)      (patch_sweep_cuda.cu:484-491) */
} efie_port_model;

typedef enum efie_scheme {
    EFIE_SCHEME_REF = 0,     /* reference quadrature: cached subdivision + softening */
    EFIE_SCHEME_EXTRACT = 1  /* regular rule everywhere + analytic 1/R extraction on
                                self and vertex-adjacent triangle pairs            */
} efie_scheme;

/* How EFIE_SOLVER_MIXED recovers the complex128 solution from the complex64
 * LU: flexible GMRES with the LU as right preconditioner (converges also
 * where u32 * cond(Z) approaches 1), or classical iterative refinement. */
typedef enum efie_refine_method {
    EFIE_REFINE_GMRES = 0,
    EFIE_REFINE_CLASSICAL = 1
} efie_refine_method;

typedef struct efie_sweep_opts {
    int32_t solver;          /* efie_solver; default EFIE_SOLVER_MIXED          */
    int32_t port_model;      /* efie_port_model; default EFIE_PORT_GAUSS        */
    int32_t scheme;          /* efie_scheme; default EFIE_SCHEME_REF            */
    double refine_tol;       /* relative residual target; default 1e-10         */
    int32_t refine_max_iter; /* default 30                                      */
    int32_t lu_nb;           /* outer LU panel width 64/128/256/512 (0 = tuned) */
    int32_t timing;          /* 1 = record per-phase CUDA-event timings         */
    int32_t batch;           /* frequencies solved together (0 = automatic: up to
                                64 from Ne 4096 on, 32 below, within 45 % of free
                                device memory)                                  */
    int32_t refine_method;   /* efie_refine_method; default EFIE_REFINE_GMRES    */
    int32_t graphs;          /* 1 (default): with timing off, the mixed LU of a
                                batch replays a CUDA graph captured on the
                                plan's first batch; 0: eager launches        */
    int32_t tile_chain;      /* complex columns of the tensor-core tile of the LU's
                                K = 64 panel-chain updates: 128 or 256 (0 = tuned) */
    int32_t tile_bulk;       /* ... of the outer panels' trailing updates (0 = tuned) */
    int32_t resident_chain;  /* 1: the K = 64 chain updates run on resident CTA pairs
                                that overlap each 256 x 128 tile's TMEM drain with the
                                next tile's MMAs (tile_chain is then unused); 0: one
                                tile per CTA pair (default)                    */
    int32_t resident_bulk;   /* 1: the outer panels' rectangular updates likewise (the
                                strip of the next panel; the symmetric factorization's
                                lower-triangle bulk stays on one tile per pair)  */
    int32_t nfreq_hint;      /* frequencies the plan's sweeps will solve (0 = unknown):
                                with batch = 0, the automatic batch is cut to the
                                balanced size for that many; efie_patch_sweep_fastquad
                                sets it to Nf                                   */
    int32_t share_factors;   /* g >= 2: with the mixed solver's coarse-to-fine
                                batches, only the first batch of each group of g is
                                factored; every frequency of the others is refined
                                (GMRES, same residual target) with the complex64
                                factors of the nearest frequency of that batch, which
                                stay in the plan's slots, and the automatic batch
                                size gives a sweep at least g batches.  1: every
                                frequency is factored.  0 (default): automatic,
                                g ~ Ne / 1200 within [2, 8] */
} efie_sweep_opts;

/* Fill `o` with the defaults listed above. */
void efie_sweep_opts_default(efie_sweep_opts *o);

/* Kernel classes of the per-launch accounting in efie_sweep_stats. */
typedef enum efie_kernel_class {
    EFIE_K_QUAD = 0,      /* regular-pair quadrature (work: point-pair evaluations) */
    EFIE_K_NEARSELF = 1,  /* near / self / singular pairs (work: point-pair evaluations) */
    EFIE_K_GATHER = 2,    /* moments -> Z entries (work: bytes of Z written) */
    EFIE_K_GEMM = 3,      /* LU trailing update (work: algorithmic real flops, 8 m n k) */
    EFIE_K_PANEL = 4,     /* LU diagonal blocks, panels, format conversion */
    EFIE_K_TRSV = 5,      /* triangular solves (work: bytes of L/U read) */
    EFIE_K_RESIDUAL = 6,  /* FP64 residual r = V - Z x (work: bytes of Z read) */
    EFIE_K_OTHER = 7,     /* port reduction, fills, complex128 LU of the FP64 path */
    EFIE_NUM_KERNEL_CLASSES = 8
} efie_kernel_class;

typedef struct efie_sweep_stats {
    int32_t n_freq;
    int32_t refine_iters_max;   /* worst-case refinement iterations over the sweep */
    int32_t n_fp64_fallback;    /* frequencies re-solved with the complex128 LU    */
    double max_relres;          /* worst final relative residual ||V - Z I||/||V|| */
    double ms_assemble;         /* summed device time per phase (timing = 1)       */
    double ms_factor;
    double ms_solve;            /* triangular solves + residuals + reduction       */
    int32_t n_launches;         /* kernels this library launched (always counted)  */
    int32_t class_launches[EFIE_NUM_KERNEL_CLASSES];
    double class_ms[EFIE_NUM_KERNEL_CLASSES];   /* summed CUDA-event time (timing = 1) */
    double class_work[EFIE_NUM_KERNEL_CLASSES]; /* summed algorithmic work, units above */
    int32_t n_wait_timeouts;    /* frequencies whose bounded device wait gave up (then
                                   re-solved by the complex128 LU)                */
    int32_t n_zero_pivots;      /* frequencies whose complex64 LU met a zero pivot */
    int32_t n_shared_factors;   /* frequencies refined with a neighbour's factors  */
} efie_sweep_stats;

/* Replaces patch_sweep_fastquad_cuda.cu:461-844 (mexFunction):
 * [Zin,S11] = patch_sweep_fastquad_cuda(V,F,E,plusTri,minusTri,plusSign,
 *     minusSign,rp,rm,Ap,Am,len,prepack,freqs,mu,eps,patchEdge,groundEdge,
 *     V0,spreadRadius,Z0).
 * opts may be NULL (defaults).  I (optional, may be NULL) receives the
 * solution currents [Ne x Nf] column-major; stats may be NULL. */
efie_status efie_patch_sweep_fastquad(efie_ctx *ctx, const efie_mesh *mesh, const efie_prepack *pre,
                                      const double *freqs, int32_t Nf, double mu, efie_c128 eps,
                                      int32_t patchEdge, int32_t groundEdge, double V0,
                                      double spreadRadius, double Z0, const efie_sweep_opts *opts,
                                      efie_c128 *Zin, efie_c128 *S11, efie_c128 *I,
                                      efie_sweep_stats *stats);

/* Replaces patch_sweep_cuda.cu:172-527 (mexFunction): centroid assembly with
 * selfAlpha fixed at 0.20 (:269) and the edge-difference port model
 * (:484-494).  opts->port_model is ignored (always EFIE_PORT_EDGE_DIFF). */
efie_status efie_patch_sweep_centroid(efie_ctx *ctx, const efie_mesh *mesh,
                                      const double *freqs, int32_t Nf, double mu, efie_c128 eps,
                                      int32_t patchEdge, int32_t groundEdge, double V0,
                                      double spreadRadius, double Z0, const efie_sweep_opts *opts,
                                      efie_c128 *Zin, efie_c128 *S11, efie_c128 *I,
                                      efie_sweep_stats *stats);

/* ---------------------------------------------------------------------- */
/* Plans: geometry uploaded once, sweeps re-run with device-resident data  */
/* ---------------------------------------------------------------------- */
typedef struct efie_plan efie_plan;

/* Upload the geometry of a patch_sweep_fastquad_cuda call once.  pre may be
 * NULL when opts->scheme == EFIE_SCHEME_EXTRACT; `rule_order` then selects the
 * regular rule (a tri_quad_rule order or EFIE_QUAD_DUNAVANT7). */
efie_status efie_plan_create(efie_ctx *ctx, const efie_mesh *mesh, const efie_prepack *pre,
                             double mu, efie_c128 eps, int32_t patchEdge, int32_t groundEdge,
                             double V0, double spreadRadius, double Z0,
                             const efie_sweep_opts *opts, int32_t rule_order, efie_plan **out);
efie_status efie_plan_run(efie_plan *plan, const double *freqs, int32_t Nf,
                          efie_c128 *Zin, efie_c128 *S11, efie_c128 *I, efie_sweep_stats *stats);
void efie_plan_destroy(efie_plan *plan);
/* Switch the per-kernel-class CUDA-event timing of later runs on (1) or off
 * (0).  Timed runs launch the factorization eagerly; untimed runs replay it
 * as a CUDA graph (opts->graphs). */
efie_status efie_plan_set_timing(efie_plan *plan, int32_t timing);

/* ---------------------------------------------------------------------- */
/* Boundary-data producers (MATLAB-side in the reference)                  */
/* ---------------------------------------------------------------------- */

/* make_patch_with_ground_mesh.m:1-46.  vertex_order 0 reproduces the
 * reference exactly (vertices numbered y-fastest by meshgrid(:), faces
 * indexed x-fastest); 1 numbers vertices x-fastest so that every face is a
 * half rectangle.  V: [Nv x 3], F: [Nt x 3] with
 * Nv = (Npx+1)(Npy+1) + (Ngx+1)(Ngy+1), Nt = 2(Npx Npy + Ngx Ngy). */
efie_status efie_make_patch_with_ground_mesh(double Lp, double Wp, double Lg, double Wg, double h,
                                             int32_t Npx, int32_t Npy, int32_t Ngx, int32_t Ngy,
                                             int32_t vertex_order, double *V, int32_t *F);

/* build_rwg_interior.m:1-103.  Call once with capacity 0 to get *Ne, then
 * again with capacity == *Ne and output arrays sized for it (column-major,
 * leading dimension Ne): edge [Ne x 2], rp/rm/center [Ne x 3]. */
efie_status efie_build_rwg_interior(int32_t Nv, const double *V, int32_t Nt, const int32_t *F,
                                    int32_t capacity, int32_t *Ne,
                                    int32_t *edge, int32_t *plusTri, int32_t *minusTri,
                                    int32_t *plusSign, int32_t *minusSign,
                                    double *rp, double *rm, double *Ap, double *Am,
                                    double *len, double *center, int32_t *zSign);

/* pick_port_edge_by_point_and_layer.m:1-11 (first minimum on ties).
 * center [Ne x 3]; returns the 1-based edge in *eidx. */
efie_status efie_pick_port_edge(int32_t Ne, const double *center, const int32_t *zSign,
                                const double p[3], int32_t layerSign, int32_t *eidx);

/* Rule selector for the Dunavant (1985) 7-point degree-5 rule, which the
 * reference lacks; every other order keeps tri_quad_rule.m's meaning
 * (1 -> 1 point, 2 -> 3 points, anything else -> the 6-point rule). */
#define EFIE_QUAD_DUNAVANT7 (-7)

/* Number of points of tri_quad_rule(order) (tri_quad_rule.m:1-23). */
int32_t efie_quad_rule_size(int32_t order);

typedef struct efie_precompute_opts {
    int32_t quad_order, near_order, self_subdiv, near_subdiv;
    double near_sing_eps, self_alpha, near_alpha;
} efie_precompute_opts;

/* efie_precompute.m:1-97 + efie_precompute_pack.m:1-59.  `out` carries the
 * dimensions (Nt, Nq = efie_quad_rule_size(quad_order), Nq2 =
 * efie_quad_rule_size(near_order), NsS = 4^self_subdiv, NsN = 4^near_subdiv)
 * and caller-allocated arrays of those sizes. */
efie_status efie_precompute_pack(int32_t Nv, const double *V, int32_t Nt, const int32_t *F,
                                 const efie_precompute_opts *opts, efie_prepack *out);

/* A two-plate design meshed and numbered on the GPU of `ctx`:
 * make_patch_with_ground_mesh.m:1-46 (same arguments and vertex_order as
 * efie_make_patch_with_ground_mesh), build_rwg_interior.m:1-113 and
 * pick_port_edge_by_point_and_layer.m:1-11 for the port edges nearest to
 * (feed[0], feed[1], +h/2) on the patch layer and (feed[0], feed[1], -h/2) on
 * the ground layer.  Every output is bit-identical to the host producers
 * (same RWG numbering, signs and port edges).  The arrays stay on the device
 * until efie_design_read copies them to caller arrays in the MEX layout
 * (sizes from efie_design_sizes; any output pointer may be NULL). */
typedef struct efie_design efie_design;
efie_status efie_design_build(efie_ctx *ctx, double Lp, double Wp, double Lg, double Wg, double h,
                              int32_t Npx, int32_t Npy, int32_t Ngx, int32_t Ngy, int32_t vertex_order,
                              const double feed[2], efie_design **out);
efie_status efie_design_sizes(const efie_design *d, int32_t *Nv, int32_t *Nt, int32_t *Ne,
                              int32_t *patchEdge, int32_t *groundEdge);
efie_status efie_design_read(const efie_design *d, double *V, int32_t *F, int32_t *edge, int32_t *plusTri,
                             int32_t *minusTri, int32_t *plusSign, int32_t *minusSign, double *rp,
                             double *rm, double *Ap, double *Am, double *len, double *center, int32_t *zSign);
void efie_design_destroy(efie_design *d);

/* The same outputs as efie_precompute_pack, computed on the GPU of `ctx`
 * from V and F (host arrays in, host arrays out; nearMat included, so
 * Nt <= 65535).  Floating-point outputs are bit-identical to the host
 * producer (every operation rounded as in efie_precompute.m, no FMA
 * contraction), and so is the uint8 nearMat. */
efie_status efie_precompute_pack_gpu(efie_ctx *ctx, int32_t Nv, const double *V, int32_t Nt, const int32_t *F,
                                     const efie_precompute_opts *opts, efie_prepack *out);

/* efie_plan_create for the reference scheme whose efie_precompute +
 * efie_precompute_pack step (efie_precompute.m:1-97,
 * efie_precompute_pack.m:1-59, MATLAB-side in the reference) runs on the
 * GPU from mesh->V and mesh->F: the quadrature caches go straight into the
 * plan's layout and the near pairs straight into its ordered pair list, so
 * the Nt x Nt nearMat is never formed on the host or sent to the device.
 * The plan is identical to one created from the host prepack of the same
 * options. */
efie_status efie_plan_create_mesh(efie_ctx *ctx, const efie_mesh *mesh, const efie_precompute_opts *popts,
                                  double mu, efie_c128 eps, int32_t patchEdge, int32_t groundEdge, double V0,
                                  double spreadRadius, double Z0, const efie_sweep_opts *opts, efie_plan **out);

/* ---------------------------------------------------------------------- */
/* Self-tests                                                              */
/* ---------------------------------------------------------------------- */

/* Factors the column-major complex128 matrix A [N x N] with the complex64
 * LU of EFIE_SOLVER_MIXED (no pivoting) and returns L (unit lower, below the
 * diagonal) and U (on and above it) packed in LU [N x N], column-major.
 * tensor_cores = 0 forces the CUDA-core trailing update.  No counterpart in
 * the reference (it calls cusolverDnZgetrf). */
efie_status efie_lu_selftest(efie_ctx *ctx, int32_t N, const efie_c128 *A, int32_t tensor_cores, efie_c128 *LU);

/* 1 disables the tensor-core trailing update process-wide (CUDA-core path). */
void efie_debug_disable_tensor_cores(int disable);

/* 1 makes the mixed LU of a symmetric Z factor it as a general matrix
 * (every trailing update over the full block) instead of L D L^T from the
 * lower part, process-wide.  Diagnostic modes: 2 keeps L D L^T but updates
 * the full trailing blocks; 3 factors the diagonal blocks as general
 * matrices (from their lower triangle) with separately inverted factors.
 * 0 restores the default.  No counterpart in the reference. */
void efie_debug_disable_symmetric_lu(int disable);

/* Outer panel width of efie_lu_selftest: 64/128/256/512 (anything else:
 * 256, the default), process-wide.  A bit-exactly symmetric A takes the
 * symmetric factorization unless efie_debug_disable_symmetric_lu(1). */
void efie_debug_set_selftest_panel(int lu_nb);

/* Test hook for the bounded device waits of the triangular solves (the
 * mixed solver's refinement), process-wide on the current device: enable = 1
 * makes every later wait target a count that no block ever publishes, so
 * each wait gives up after `spins` polls, records a timeout for its frequency
 * and returns; those frequencies are re-solved by the complex128 LU and
 * counted in efie_sweep_stats.n_wait_timeouts.  enable = 0 restores the
 * production limit (2^23 polls, about a second).  No counterpart in the
 * reference. */
efie_status efie_debug_set_wait_test(int32_t enable, int64_t spins);

/* Tensor-core tile widths (128 or 256 complex columns per CTA pair; anything
 * else: 256) of efie_lu_selftest's K = 64 chain updates and outer-panel
 * updates, and which of them run on resident CTA pairs (bit 0: the chain's,
 * bit 1: the outer panels'; efie_sweep_opts.resident_chain / resident_bulk),
 * process-wide.  No counterpart in the reference. */
void efie_debug_set_selftest_tiles(int tile_chain, int tile_bulk, int resident);

/* 1 makes efie_plan_run take its batches in frequency order with every
 * refinement starting from zero, instead of coarse to fine with initial
 * guesses interpolated from the solved neighbours (mixed solver, GMRES, more
 * than one batch), process-wide.  No counterpart in the reference. */
void efie_debug_disable_warm_start(int disable);

/* ---------------------------------------------------------------------- */
/* Centroid assembly without device allocation                             */
/* ---------------------------------------------------------------------- */
#define EFIE_NOALLOC_MAX_NE 16384
#define EFIE_NOALLOC_MAX_NT 16384

/* No counterpart in the reference.  The same result as efie_gassemble_zv
 * (Z and Vrhs of the one-point centroid assembly) for callers that cannot
 * call cudaMalloc -- processes held to a device-memory budget fixed at
 * start-up, hosts that own every device buffer and do not let a library
 * allocate.  Every array argument (V ... len, Z, Vrhs) is a DEVICE pointer in
 * the MEX layout; exc (host) = [patchEdge, groundEdge, V0, spreadRadius,
 * selfAlpha].  The function allocates nothing: its scratch is one fixed
 * __device__ array (about 3.2 MB) that every GPU loading this library keeps
 * until exit, which limits Ne <= EFIE_NOALLOC_MAX_NE and Nt <=
 * EFIE_NOALLOC_MAX_NT (larger sizes are rejected with EFIE_ERR_ARGS).  All
 * calls share that array: calls that overlap on the GPU race, so serialise
 * them.  The first call on a device looks up the array's address with that
 * device current and keeps it for the life of the process: make it before
 * any stream capture, and do not call this function across a cudaDeviceReset
 * of that device.  Runs on `stream` (a cudaStream_t) and returns after
 * synchronising it.  Index errors that only the device sees (F, E,
 * plusTri/minusTri out of range, no Gaussian port weights) return mex:F,
 * mex:E, mex:rwg and mex:rhs without touching out-of-range memory. */
efie_status efie_gassemble_zv_noalloc(int device, void *stream, int32_t Nv, int32_t Nt, int32_t Ne,
                                      const double *V, const int32_t *F, const int32_t *E,
                                      const int32_t *plusTri, const int32_t *minusTri,
                                      const int32_t *plusSign, const int32_t *minusSign,
                                      const double *rp, const double *rm, const double *Ap, const double *Am,
                                      const double *len, efie_c128 k, double omega, double mu, efie_c128 eps,
                                      const double exc[5], efie_c128 *Z, efie_c128 *Vrhs);

/* ---------------------------------------------------------------------- */
/* Surrogate MLP for adaptive sweeps                                       */
/* ---------------------------------------------------------------------- */
/* No counterpart in the reference.  A multilayer perceptron from normalised
 * (geometry, frequency) features to the normalised Zin, trained and evaluated
 * by the library's own CUDA kernels: n_layers hidden layers of width n_hidden
 * with SiLU, a linear output layer; BF16 weight matrices with FP32
 * accumulation in every layer, FP32 biases, activations and gradients, Adam
 * on FP32 master weights.  One training step (minibatch gather, forward, MSE
 * loss, backward, Adam) runs as one captured CUDA graph.
 *
 * Parameter vector (get/set_params, loss_grad): for each linear layer
 * l = 0..n_layers, W_l [out_l x in_l] row-major then b_l [out_l]; in_0 = n_in,
 * out_{n_layers} = n_out, every other width n_hidden.  X is [n x n_in] and
 * T, Y are [n x n_out], row-major FP32 host arrays. */
#define EFIE_MLP_MAX_LAYERS 8

typedef struct efie_mlp efie_mlp;

typedef struct efie_mlp_config {
    int32_t n_in;       /* default 5: W, L, h, feed offset, frequency */
    int32_t n_hidden;   /* default 256 */
    int32_t n_layers;   /* hidden layers, default 4 (<= EFIE_MLP_MAX_LAYERS) */
    int32_t n_out;      /* default 2: Re, Im */
    uint64_t seed;      /* initial weights: uniform(-1/sqrt(in), 1/sqrt(in)) */
} efie_mlp_config;

typedef struct efie_adam_opts {
    float lr, beta1, beta2, eps, weight_decay;   /* 1e-3, 0.9, 0.999, 1e-8, 0 */
    int32_t batch;                               /* minibatch rows, default 1024 */
    int32_t epochs;                              /* default 100 */
    uint64_t seed;                               /* minibatch shuffling */
} efie_adam_opts;

void efie_mlp_config_default(efie_mlp_config *cfg);
void efie_adam_opts_default(efie_adam_opts *opts);
efie_status efie_mlp_create(efie_ctx *ctx, const efie_mlp_config *cfg, efie_mlp **out);
void efie_mlp_destroy(efie_mlp *mlp);
int64_t efie_mlp_num_params(const efie_mlp *mlp);
efie_status efie_mlp_get_params(efie_mlp *mlp, float *params);
/* Also resets Adam's moments and step count. */
efie_status efie_mlp_set_params(efie_mlp *mlp, const float *params);
efie_status efie_mlp_forward(efie_mlp *mlp, const float *X, int32_t n, float *Y);
/* loss = mean over the n x n_out entries of (Y - T)^2 and its gradient with
 * respect to the parameter vector (either output may be NULL). */
efie_status efie_mlp_loss_grad(efie_mlp *mlp, const float *X, const float *T, int32_t n, double *loss,
                               float *grad);
/* opts->epochs passes over the n samples in shuffled minibatches of
 * opts->batch rows (floor(n / batch) per epoch); loss_history (may be NULL)
 * receives each epoch's mean minibatch loss. */
efie_status efie_mlp_train(efie_mlp *mlp, const float *X, const float *T, int32_t n, const efie_adam_opts *opts,
                           double *loss_history);

#ifdef __cplusplus
}
#endif
#endif /* EFIE_B200_H */
