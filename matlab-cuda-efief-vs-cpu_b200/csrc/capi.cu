// C ABI of libefie_b200: argument checks that mirror the reference MEX
// functions, host-side RHS, plans and frequency sweeps.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <map>
#include <mutex>
#include <vector>

#include "efie_internal.h"
#include "solve.h"

namespace {
thread_local std::string g_last_error;
}

efie_status efie_fail(efie_status s, const std::string &msg) {
    g_last_error = msg;
    return s;
}

extern "C" const char *efie_last_error(void) { return g_last_error.c_str(); }

extern "C" const char *efie_status_id(efie_status s) {
    switch (s) {
    case EFIE_OK: return "";
    case EFIE_ERR_ARGS: return "mex:args";
    case EFIE_ERR_V: return "mex:V";
    case EFIE_ERR_F: return "mex:F";
    case EFIE_ERR_E: return "mex:E";
    case EFIE_ERR_RWG: return "mex:rwg";
    case EFIE_ERR_PORT: return "mex:port";
    case EFIE_ERR_PREPACK: return "mex:prepack";
    case EFIE_ERR_R_REG: return "mex:r_reg";
    case EFIE_ERR_W_REG: return "mex:w_reg";
    case EFIE_ERR_NEARMAT: return "mex:nearMat";
    case EFIE_ERR_SELF_R: return "mex:self_r";
    case EFIE_ERR_SELF_W: return "mex:self_w";
    case EFIE_ERR_SELF_A: return "mex:self_a";
    case EFIE_ERR_NEAR_R: return "mex:near_r";
    case EFIE_ERR_NEAR_W: return "mex:near_w";
    case EFIE_ERR_AEQTRI: return "mex:aeqTri";
    case EFIE_ERR_RHS: return "mex:rhs";
    case EFIE_ERR_EPS: return "mex:eps";
    case EFIE_ERR_EXC: return "mex:exc";
    case EFIE_ERR_FREQS: return "mex:freqs";
    case EFIE_ERR_CUDA: return "cuda:rt";
    case EFIE_ERR_CUSOLVER: return "cuda:cusolver";
    case EFIE_ERR_SINGULAR: return "efie:singular";
    case EFIE_ERR_NOMEM: return "efie:nomem";
    case EFIE_ERR_TIMEOUT: return "efie:timeout";
    case EFIE_ERR_MESH: return "efie:mesh";
    }
    return "efie:unknown";
}

extern "C" void efie_sweep_opts_default(efie_sweep_opts *o) {
    if (!o) return;
    o->solver = EFIE_SOLVER_MIXED;
    o->port_model = EFIE_PORT_GAUSS;
    o->scheme = EFIE_SCHEME_REF;
    o->refine_tol = 1e-10;
    o->refine_max_iter = 30;
    o->refine_method = EFIE_REFINE_GMRES;
    o->graphs = 1;
    o->lu_nb = 0;
    o->timing = 0;
    o->batch = 0;
    o->tile_chain = 0;
    o->tile_bulk = 0;
    o->resident_chain = 0;
    o->resident_bulk = 0;
    o->nfreq_hint = 0;
    o->share_factors = 0;
}

// ---------------------------------------------------------------------------
// Context
// ---------------------------------------------------------------------------
extern "C" efie_status efie_ctx_create(int device, efie_ctx **out) {
    if (!out) return efie_fail(EFIE_ERR_ARGS, "efie_ctx_create: null output");
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n <= device || device < 0)
        return efie_fail(EFIE_ERR_CUDA, std::string("no CUDA device ") + std::to_string(device) + ": " +
                                            (e == cudaSuccess ? "out of range" : cudaGetErrorString(e)));
    EFIE_CUDA(cudaSetDevice(device));
    efie_ctx *c = new (std::nothrow) efie_ctx();
    if (!c) return efie_fail(EFIE_ERR_NOMEM, "efie_ctx_create: out of host memory");
    c->device = device;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
        delete c;
        return efie_fail(EFIE_ERR_CUDA, "cudaGetDeviceProperties failed");
    }
    c->num_sms = prop.multiProcessorCount;
    c->cc_major = prop.major;
    if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return efie_fail(EFIE_ERR_CUDA, "cudaStreamCreate failed");
    }
    c->stream = c->own_stream;
    if (cusolverDnCreate(&c->solver) != CUSOLVER_STATUS_SUCCESS) {
        cudaStreamDestroy(c->own_stream);
        delete c;
        return efie_fail(EFIE_ERR_CUSOLVER, "cusolverDnCreate failed");
    }
    cusolverDnSetStream(c->solver, c->stream);
    *out = c;
    return EFIE_OK;
}

extern "C" void efie_ctx_destroy(efie_ctx *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->solver) cusolverDnDestroy(ctx->solver);
    ctx->status.release();
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    efie_pool_trim(ctx->device);
    delete ctx;
}

namespace {

struct DevicePool {
    std::multimap<size_t, void *> free;   // size -> block
    size_t cached = 0;
    size_t cap = 0;
};

std::mutex g_pool_mu;
// never destroyed: cached blocks are left to the driver at process exit
std::map<int, DevicePool> *g_pools = new std::map<int, DevicePool>();

DevicePool &pool_of(int dev) {
    DevicePool &P = (*g_pools)[dev];
    if (!P.cap) {
        size_t fr = 0, total = 0;
        if (cudaMemGetInfo(&fr, &total) == cudaSuccess) P.cap = total / 10 * 4;
        else P.cap = 1;
    }
    return P;
}

void trim_locked(DevicePool &P) {
    for (auto &kv : P.free) cudaFree(kv.second);
    P.free.clear();
    P.cached = 0;
}

}  // namespace

void *efie_pool_get(size_t n, size_t *got, cudaError_t *err) {
    int dev = 0;
    cudaGetDevice(&dev);
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        DevicePool &P = pool_of(dev);
        auto it = P.free.lower_bound(n);
        if (it != P.free.end() && it->first <= 2 * n) {
            void *p = it->second;
            *got = it->first;
            P.cached -= it->first;
            P.free.erase(it);
            return p;
        }
    }
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, n);
    if (e != cudaSuccess) {
        cudaGetLastError();   // clear the sticky-free allocation error
        {
            std::lock_guard<std::mutex> lk(g_pool_mu);
            trim_locked(pool_of(dev));
        }
        e = cudaMalloc(&p, n);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (err) *err = e;
        return nullptr;
    }
    *got = n;
    return p;
}

void efie_pool_put(void *p, size_t bytes) {
    // the block's last users may still run: finish them as cudaFree would
    cudaDeviceSynchronize();
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_pool_mu);
    DevicePool &P = pool_of(dev);
    if (bytes > P.cap) {
        cudaFree(p);
        return;
    }
    P.free.emplace(bytes, p);
    P.cached += bytes;
    while (P.cached > P.cap && !P.free.empty()) {   // drop the largest blocks first
        auto it = std::prev(P.free.end());
        cudaFree(it->second);
        P.cached -= it->first;
        P.free.erase(it);
    }
}

void efie_pool_trim(int device) {
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        trim_locked(pool_of(device));
    }
    cudaSetDevice(prev);
}

size_t efie_pool_cached(int device) {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    auto it = g_pools->find(device);
    return it == g_pools->end() ? 0 : it->second.cached;
}

extern "C" efie_status efie_ctx_set_stream(efie_ctx *ctx, void *stream) {
    if (!ctx) return efie_fail(EFIE_ERR_ARGS, "null context");
    ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
    if (cusolverDnSetStream(ctx->solver, ctx->stream) != CUSOLVER_STATUS_SUCCESS)
        return efie_fail(EFIE_ERR_CUSOLVER, "cusolverDnSetStream failed");
    return EFIE_OK;
}

// ---------------------------------------------------------------------------
// Argument checks (the reference's mexErrMsgIdAndTxt identifiers)
// ---------------------------------------------------------------------------
namespace {

efie_status check_mesh(const efie_mesh *m, bool need_E) {
    if (!m) return efie_fail(EFIE_ERR_ARGS, "null mesh");
    if (!m->V || m->Nv < 1) return efie_fail(EFIE_ERR_V, "V must be [Nv x 3] double.");
    if (!m->F || m->Nt < 1) return efie_fail(EFIE_ERR_F, "F must be [Nt x 3] int32.");
    if (m->Ne < 0 || (need_E && !m->E)) return efie_fail(EFIE_ERR_E, "E must be [Ne x 2] int32.");
    if (m->Ne > 0 && (!m->plusTri || !m->minusTri || !m->plusSign || !m->minusSign || !m->rp || !m->rm ||
                      !m->Ap || !m->Am || !m->len))
        return efie_fail(EFIE_ERR_RWG, "missing RWG arrays.");
    for (int64_t i = 0; i < 3 * (int64_t)m->Nt; i++)
        if (m->F[i] < 1 || m->F[i] > m->Nv) return efie_fail(EFIE_ERR_F, "F has invalid indices.");
    if (need_E)
        for (int64_t i = 0; i < 2 * (int64_t)m->Ne; i++)
            if (m->E[i] < 1 || m->E[i] > m->Nv) return efie_fail(EFIE_ERR_E, "E has invalid indices.");
    for (int e = 0; e < m->Ne; e++) {
        if (m->plusTri[e] < 0 || m->plusTri[e] > m->Nt || m->minusTri[e] < 0 || m->minusTri[e] > m->Nt)
            return efie_fail(EFIE_ERR_RWG, "plusTri/minusTri out of range.");
        if ((m->plusTri[e] > 0 && !(m->Ap[e] != 0.0)) || (m->minusTri[e] > 0 && !(m->Am[e] != 0.0)))
            return efie_fail(EFIE_ERR_RWG, "Ap/Am must be nonzero on supported triangles.");
    }
    return EFIE_OK;
}

efie_status check_prepack(const efie_mesh *m, const efie_prepack *p) {
    if (!p) return efie_fail(EFIE_ERR_PREPACK, "prepack must be a struct from efie_precompute_pack.");
    if (!p->r_reg || p->Nq < 1) return efie_fail(EFIE_ERR_R_REG, "r_reg must be [Nq x 3 x Nt] double.");
    if (!p->w_reg) return efie_fail(EFIE_ERR_W_REG, "w_reg must be [Nq x Nt] double.");
    if (!p->nearMat) return efie_fail(EFIE_ERR_NEARMAT, "nearMat must be uint8 [Nt x Nt].");
    if (!p->self_r || p->Nq2 < 1 || p->NsS < 1) return efie_fail(EFIE_ERR_SELF_R, "self_r must be [Nq2 x 3 x NsS x Nt].");
    if (!p->self_w) return efie_fail(EFIE_ERR_SELF_W, "self_w must be [Nq2 x NsS x Nt].");
    if (!p->self_a) return efie_fail(EFIE_ERR_SELF_A, "self_a must be [NsS x Nt].");
    if (!p->near_r || p->NsN < 1) return efie_fail(EFIE_ERR_NEAR_R, "near_r must be [Nq2 x 3 x NsN x Nt].");
    if (!p->near_w) return efie_fail(EFIE_ERR_NEAR_W, "near_w must be [Nq2 x NsN x Nt].");
    if (!p->aeqTri || p->Nt != m->Nt) return efie_fail(EFIE_ERR_AEQTRI, "aeqTri must be [Nt x 1].");
    return EFIE_OK;
}

// build_Vrhs_gaussian (ggassemble_ZV_EFIE_RWG_DIFF_GPU_FAST.cu:492-540) /
// build_weights_gaussian (patch_sweep_fastquad_cuda.cu:415-459), FP64 on the host.
efie_status gauss_weights(const efie_mesh *m, int edge1, double spread, std::vector<double> &w) {
    const int Ne = m->Ne, Nv = m->Nv;
    std::vector<double> cx(Ne), cy(Ne), cz(Ne);
    double zmin = 1e100, zmax = -1e100;
    for (int e = 0; e < Ne; e++) {
        const int a = m->E[e] - 1, b = m->E[e + Ne] - 1;
        cx[e] = 0.5 * (m->V[a] + m->V[b]);
        cy[e] = 0.5 * (m->V[a + Nv] + m->V[b + Nv]);
        cz[e] = 0.5 * (m->V[a + 2 * (size_t)Nv] + m->V[b + 2 * (size_t)Nv]);
        zmin = std::min(zmin, cz[e]);
        zmax = std::max(zmax, cz[e]);
    }
    const double zmid = 0.5 * (zmin + zmax);
    const int e0 = edge1 - 1;
    const int layer0 = cz[e0] > zmid ? 1 : -1;
    w.assign(Ne, 0.0);
    double sumw = 0.0;
    for (int e = 0; e < Ne; e++) {
        const int layer = cz[e] > zmid ? 1 : -1;
        if (layer != layer0) continue;
        const double dx = cx[e] - cx[e0], dy = cy[e] - cy[e0], dz = cz[e] - cz[e0];
        const double dist = std::sqrt(dx * dx + dy * dy + dz * dz);
        const double v = std::exp(-(dist / spread) * (dist / spread));
        w[e] = v;
        sumw += v;
    }
    if (!(sumw >= 1e-30)) return efie_fail(EFIE_ERR_RHS, "spreadRadius too small (no weights).");
    for (int e = 0; e < Ne; e++) w[e] /= sumw;
    return EFIE_OK;
}

efie_status build_rhs(const efie_mesh *m, int pe, int ge, double V0, double spread, std::vector<double> &rhs,
                      std::vector<double> *wport) {
    std::vector<double> wP, wG;
    EFIE_TRY(gauss_weights(m, pe, spread, wP));
    EFIE_TRY(gauss_weights(m, ge, spread, wG));
    rhs.resize(m->Ne);
    for (int e = 0; e < m->Ne; e++) rhs[e] = (+V0 / 2.0) * wP[e] + (-V0 / 2.0) * wG[e];
    if (wport) {
        wport->resize(m->Ne);
        for (int e = 0; e < m->Ne; e++) (*wport)[e] = (wP[e] - wG[e]) * m->len[e];  // fastquad.cu:780
    }
    return EFIE_OK;
}

efie_status check_port(const efie_mesh *m, int pe, int ge) {
    if (!(pe >= 1 && pe <= m->Ne)) return efie_fail(EFIE_ERR_PORT, "patchEdge out of range.");
    if (!(ge >= 1 && ge <= m->Ne)) return efie_fail(EFIE_ERR_PORT, "groundEdge out of range.");
    return EFIE_OK;
}

efie_status check_eps(double omega, efie_c128 eps) {
    const double dr = -omega * eps.im, di = omega * eps.re;
    if (!(dr * dr + di * di > 0.0)) return efie_fail(EFIE_ERR_EPS, "eps causes denom=0.");
    return EFIE_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// Assembly-only entry points
// ---------------------------------------------------------------------------
extern "C" efie_status efie_ggassemble_zv(efie_ctx *ctx, const efie_mesh *mesh, const efie_prepack *pre,
                                          efie_c128 k, double omega, double mu, efie_c128 eps,
                                          const double excvec[4], efie_c128 *Z, efie_c128 *Vrhs) {
    if (!ctx) return efie_fail(EFIE_ERR_ARGS, "null context");
    EFIE_TRY(check_mesh(mesh, true));
    EFIE_TRY(check_prepack(mesh, pre));
    if (!excvec) return efie_fail(EFIE_ERR_EXC, "excvec must be [patchEdge, groundEdge, V0, spreadRadius].");
    const int pe = (int)excvec[0], ge = (int)excvec[1];
    EFIE_TRY(check_port(mesh, pe, ge));
    if (!Z || !Vrhs) return efie_fail(EFIE_ERR_ARGS, "null output");
    DeviceGuard dg(ctx->device);
    std::vector<double> rhs;
    EFIE_TRY(build_rhs(mesh, pe, ge, excvec[2], excvec[3], rhs, nullptr));
    EFIE_TRY(check_eps(omega, eps));
    const Physics ph = efie_physics_k(k, omega, mu, eps);
    const int Ne = mesh->Ne;
    GeomDev g;
    EFIE_TRY(efie_geom_upload(ctx, mesh, pre, EFIE_SCHEME_REF, 0, g));
    DevBuf dZ;
    EFIE_TRY(dZ.reserve(sizeof(efie_c128) * (size_t)Ne * Ne));
    EFIE_TRY(efie_assemble_device(ctx, g, ph, dZ.p));
    EFIE_CUDA(cudaMemcpyAsync(Z, dZ.p, sizeof(efie_c128) * (size_t)Ne * Ne, cudaMemcpyDeviceToHost, ctx->stream));
    EFIE_CUDA(cudaStreamSynchronize(ctx->stream));
    for (int e = 0; e < Ne; e++) Vrhs[e] = efie_c128{rhs[e], 0.0};
    return EFIE_OK;
}

extern "C" efie_status efie_gassemble_zv(efie_ctx *ctx, const efie_mesh *mesh, efie_c128 k, double omega, double mu,
                                         efie_c128 eps, const double exc[5], efie_c128 *Z, efie_c128 *Vrhs) {
    if (!ctx) return efie_fail(EFIE_ERR_ARGS, "null context");
    EFIE_TRY(check_mesh(mesh, true));
    if (!exc)
        return efie_fail(EFIE_ERR_EXC,
                         "exc must be double vector len>=5: [patchEdge, groundEdge, V0, spreadRadius, selfAlpha].");
    const int pe = (int)exc[0], ge = (int)exc[1];
    EFIE_TRY(check_port(mesh, pe, ge));
    if (!Z || !Vrhs) return efie_fail(EFIE_ERR_ARGS, "null output");
    DeviceGuard dg(ctx->device);
    std::vector<double> rhs;
    EFIE_TRY(build_rhs(mesh, pe, ge, exc[2], exc[3], rhs, nullptr));
    const Physics ph = efie_physics_k(k, omega, mu, eps);
    const int Ne = mesh->Ne;
    DevBuf dZ, scratch;
    EFIE_TRY(dZ.reserve(sizeof(efie_c128) * (size_t)Ne * Ne));
    EFIE_TRY(efie_assemble_centroid_device(ctx, mesh, exc[4], ph, dZ.p, scratch));
    EFIE_CUDA(cudaMemcpyAsync(Z, dZ.p, sizeof(efie_c128) * (size_t)Ne * Ne, cudaMemcpyDeviceToHost, ctx->stream));
    EFIE_CUDA(cudaStreamSynchronize(ctx->stream));
    for (int e = 0; e < Ne; e++) Vrhs[e] = efie_c128{rhs[e], 0.0};
    return EFIE_OK;
}

// ---------------------------------------------------------------------------
// Plans and sweeps
// ---------------------------------------------------------------------------
struct efie_plan {
    efie_ctx *ctx = nullptr;
    DevBuf rs_info;              // cuSOLVER getrs status (argument errors only)
    efie_sweep_opts opts;
    bool centroid = false;       // patch_sweep_cuda model
    double self_alpha = 0.20;
    int Ne = 0;
    int B = 1;                   // frequencies per batch
    int share_group = 1;         // batches per factored batch (1: every frequency factored)
    double mu = 0, V0 = 0, Z0 = 0;
    efie_c128 eps{0, 0};
    int pe = 0, ge = 0;
    double bnorm = 0;
    GeomDev g;
    // centroid path keeps the host mesh arrays it needs
    std::vector<double> hV, hrp, hrm, hAp, hAm, hlen;
    std::vector<int32_t> hF, hpt, hmt, hps, hms;
    efie_mesh cmesh{};
    DevBuf Z, b, x, wport, out, scratch, ipiv, info, lwork;
    DevBuf xall;   // solutions of a sweep by sorted frequency (initial guesses of later batches)
    int lwork_elems = -1;
    SolveWork sw;
    // the mixed factorization as a CUDA graph (captured on the first untimed
    // batch, replayed for every later one) and its per-class launch counts
    cudaGraphExec_t factor_graph = nullptr;
    int graph_launches[EFIE_NUM_KERNEL_CLASSES] = {0};
    double graph_work[EFIE_NUM_KERNEL_CLASSES] = {0};
    ~efie_plan() {
        if (factor_graph) cudaGraphExecDestroy(factor_graph);
    }
};

namespace {

// The mixed factorization of one batch.  With timing off (and graphs not
// disabled) the kernel sequence -- about 4 launches per 64-column block, all
// with fixed arguments for a given plan -- is captured once and replayed as a
// CUDA graph; with timing on it runs eagerly so each launch keeps its events.
efie_status plan_factor(efie_plan *p, const int *active, int nact) {
    efie_ctx *ctx = p->ctx;
    const size_t NN = (size_t)p->Ne * p->Ne;
    EFIE_TRY(efie_mixed_factor_prepare(ctx, p->sw, active));
    // the legacy default stream cannot be captured: launch eagerly there
    const bool graph = !ctx->log.timing && p->opts.graphs && ctx->stream != nullptr;
    if (!graph) return efie_mixed_factor_launch(ctx, p->sw, p->Z.p, NN, nact);
    KernelLog &log = ctx->log;
    if (!p->factor_graph) {
        int l0[EFIE_NUM_KERNEL_CLASSES];
        double w0[EFIE_NUM_KERNEL_CLASSES];
        for (int c = 0; c < EFIE_NUM_KERNEL_CLASSES; c++) l0[c] = log.launches[c], w0[c] = log.work[c];
        cudaGraph_t g = nullptr;
        EFIE_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        // the captured sequence works on every slot; `active` (device) gates them
        efie_status st = efie_mixed_factor_launch(ctx, p->sw, p->Z.p, NN, p->B);
        cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
        if (st != EFIE_OK) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        // keep the priorities of the capturing streams (the panel chain ahead of
        // the bulk trailing updates) in the replayed graph
        if (e == cudaSuccess)
            e = cudaGraphInstantiateWithFlags(&p->factor_graph, g, cudaGraphInstantiateFlagUseNodePriority);
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            p->factor_graph = nullptr;
            return efie_fail(EFIE_ERR_CUDA, std::string("factor graph: ") + cudaGetErrorString(e));
        }
        for (int c = 0; c < EFIE_NUM_KERNEL_CLASSES; c++) {
            p->graph_launches[c] = log.launches[c] - l0[c];
            p->graph_work[c] = (log.work[c] - w0[c]) * nact / std::max(1, p->B);
            log.launches[c] = l0[c];
            log.work[c] = w0[c];
        }
    }
    EFIE_CUDA(cudaGraphLaunch(p->factor_graph, ctx->stream));
    for (int c = 0; c < EFIE_NUM_KERNEL_CLASSES; c++) {
        log.launches[c] += p->graph_launches[c];
        log.work[c] += p->graph_work[c];
    }
    return EFIE_OK;
}

// complex128 LU (cuSOLVER) of Z_f in place and x_f = Z_f^-1 V
efie_status plan_solve_fp64(efie_plan *p, int slot, int fi) {
    efie_ctx *ctx = p->ctx;
    const int N = p->Ne;
    cuDoubleComplex *A = p->Z.as<cuDoubleComplex>() + (size_t)N * N * slot;
    cuDoubleComplex *x = p->x.as<cuDoubleComplex>() + (size_t)N * slot;
    if (p->lwork_elems < 0) {
        int lw = 0;
        if (cusolverDnZgetrf_bufferSize(ctx->solver, N, N, A, N, &lw) != CUSOLVER_STATUS_SUCCESS)
            return efie_fail(EFIE_ERR_CUSOLVER, "cuSOLVER error");
        EFIE_TRY(p->lwork.reserve(sizeof(cuDoubleComplex) * (size_t)std::max(lw, 1)));
        p->lwork_elems = lw;
    }
    EFIE_CUDA(cudaMemcpyAsync(x, p->b.p, sizeof(cuDoubleComplex) * N, cudaMemcpyDeviceToDevice, ctx->stream));
    // getrf's info (a zero pivot: efie:singular) in slot fi; getrs reports
    // only argument errors, into a slot of its own so that it cannot
    // overwrite getrf's
    EFIE_TRY(p->rs_info.reserve(sizeof(int)));
    int *dinfo = p->info.as<int>() + fi;
    if (cusolverDnZgetrf(ctx->solver, N, N, A, N, p->lwork.as<cuDoubleComplex>(), p->ipiv.as<int>(), dinfo) !=
        CUSOLVER_STATUS_SUCCESS)
        return efie_fail(EFIE_ERR_CUSOLVER, "cuSOLVER error");
    if (cusolverDnZgetrs(ctx->solver, CUBLAS_OP_N, N, 1, A, N, p->ipiv.as<int>(), x, N, p->rs_info.as<int>()) !=
        CUSOLVER_STATUS_SUCCESS)
        return efie_fail(EFIE_ERR_CUSOLVER, "cuSOLVER error");
    return EFIE_OK;
}

// Frequencies per batch: everything a frequency needs on the device (Z in
// complex128, its complex64 planes, staging) within a fraction of free HBM,
// at most 64 frequencies from Ne 4096 on (where the LU's panel chain is long
// enough that paying it for fewer batches wins) and 32 below (where more,
// smaller batches give more warm-started GMRES runs).  With the number of
// frequencies a sweep will solve (nf > 0), the slots are cut to the balanced
// batch size of that many batches: no slot stays idle.
// Batches per factored batch with shared factors: the caller's g >= 2, 1 for
// none, else (0) automatic.  A factorization costs O(N^3) and the GMRES steps
// it saves O(N^2) each, so larger problems share each factorization among
// more frequencies: measured on one B200, 6 is best at N 6968 (347 against
// 333 for 4 and 323 for 8 points/s) and 8 at N 19936 (36.2 against 29.3
// for 4), so g ~ N / 1200 within [2, 8].
int choose_share_group(int N, int requested) {
    if (requested == 1) return 1;
    if (requested >= 2) return std::min(requested, 16);
    return std::max(2, std::min(8, (int)std::lround(N / 1200.0)));
}

// group: batches per factored batch with shared factors (> 1): a sweep of nf
// frequencies then has at least that many batches
int choose_batch(int N, int requested, int solver, int nf, int group = 1) {
    if (solver == EFIE_SOLVER_FP64) return 1;
    if (requested > 0) return std::min(requested, EFIE_MAX_BATCH);
    size_t freeb = 0, total = 0;
    if (cudaMemGetInfo(&freeb, &total) != cudaSuccess) return 1;
    int dev = 0;
    cudaGetDevice(&dev);
    freeb += efie_pool_cached(dev);   // cached blocks are available to this plan
    const double per = 26.0 * (double)N * N + 1e6;
    int B = (int)std::floor(0.45 * (double)freeb / per);
    B = std::max(1, std::min(B, N >= 4096 ? EFIE_MAX_BATCH : 32));
    if (nf > 0) {
        const int nbat = std::max((nf + B - 1) / B, std::min(std::max(group, 1), nf));
        B = (nf + nbat - 1) / nbat;
    }
    return B;
}

// Outer LU panel width: the caller's choice, else the tuned table (wider
// panels cut trailing-matrix traffic; narrower ones keep fewer terms per
// tensor-core accumulation).
int choose_panel(int N, int requested) {
    if (requested == 64 || requested == 128 || requested == 256 || requested == 512) return requested;
    return N >= 4096 ? 512 : 128;
}

// Tile width (complex columns per CTA pair) of the tensor-core updates: the
// caller's (tuned) choice, else 256.
int choose_tile(int requested) { return requested == 128 ? 128 : 256; }

efie_status plan_common(efie_plan *p, const efie_mesh *mesh, double mu, efie_c128 eps, int pe, int ge, double V0,
                        double spread, double Z0, const efie_sweep_opts *opts) {
    efie_ctx *ctx = p->ctx;
    if (opts) p->opts = *opts;
    else efie_sweep_opts_default(&p->opts);
    if (p->opts.solver != EFIE_SOLVER_FP64 && p->opts.solver != EFIE_SOLVER_MIXED)
        return efie_fail(EFIE_ERR_ARGS, "unknown solver");
    if (!(p->opts.refine_tol > 0)) p->opts.refine_tol = 1e-10;
    if (p->opts.refine_max_iter <= 0) p->opts.refine_max_iter = 30;
    if (p->opts.refine_method != EFIE_REFINE_GMRES && p->opts.refine_method != EFIE_REFINE_CLASSICAL)
        return efie_fail(EFIE_ERR_ARGS, "unknown refinement method");
    EFIE_TRY(check_port(mesh, pe, ge));
    const int N = mesh->Ne;
    p->Ne = N;
    p->mu = mu;
    p->eps = eps;
    p->pe = pe;
    p->ge = ge;
    p->V0 = V0;
    p->Z0 = Z0;
    std::vector<double> rhs, wport;
    EFIE_TRY(build_rhs(mesh, pe, ge, V0, spread, rhs, &wport));
    std::vector<efie_c128> bc(N);
    double bn = 0;
    for (int e = 0; e < N; e++) {
        bc[e] = efie_c128{rhs[e], 0.0};
        bn += rhs[e] * rhs[e];
    }
    p->bnorm = std::sqrt(bn);
    p->share_group = p->opts.solver == EFIE_SOLVER_MIXED && p->opts.refine_method == EFIE_REFINE_GMRES
                         ? choose_share_group(N, p->opts.share_factors)
                         : 1;
    p->B = choose_batch(N, p->opts.batch, p->opts.solver, p->opts.nfreq_hint, p->share_group);
    EFIE_TRY(p->Z.reserve(sizeof(efie_c128) * (size_t)N * N * p->B));
    EFIE_TRY(p->b.reserve(sizeof(efie_c128) * N));
    EFIE_TRY(p->x.reserve(sizeof(efie_c128) * (size_t)N * p->B));
    EFIE_TRY(p->wport.reserve(sizeof(double) * N));
    EFIE_TRY(p->ipiv.reserve(sizeof(int) * N));
    EFIE_CUDA(cudaMemcpyAsync(p->b.p, bc.data(), sizeof(efie_c128) * N, cudaMemcpyHostToDevice, ctx->stream));
    EFIE_CUDA(cudaMemcpyAsync(p->wport.p, wport.data(), sizeof(double) * N, cudaMemcpyHostToDevice, ctx->stream));
    if (p->opts.solver == EFIE_SOLVER_MIXED) {
        EFIE_TRY(efie_mixed_workspace(p->sw, N, p->B, choose_panel(N, p->opts.lu_nb)));
        p->sw.tn_chain = choose_tile(p->opts.tile_chain);
        p->sw.tn_bulk = choose_tile(p->opts.tile_bulk);
        p->sw.resident_chain = p->opts.resident_chain == 1;
        p->sw.resident_bulk = p->opts.resident_bulk == 1;
    }
    EFIE_CUDA(cudaStreamSynchronize(ctx->stream));
    return EFIE_OK;
}

}  // namespace

extern "C" efie_status efie_plan_create(efie_ctx *ctx, const efie_mesh *mesh, const efie_prepack *pre, double mu,
                                        efie_c128 eps, int32_t patchEdge, int32_t groundEdge, double V0,
                                        double spreadRadius, double Z0, const efie_sweep_opts *opts,
                                        int32_t rule_order, efie_plan **out) {
    if (!ctx || !out) return efie_fail(EFIE_ERR_ARGS, "null context or output");
    *out = nullptr;
    EFIE_TRY(check_mesh(mesh, true));
    const int scheme = opts ? opts->scheme : EFIE_SCHEME_REF;
    if (scheme == EFIE_SCHEME_REF) EFIE_TRY(check_prepack(mesh, pre));
    DeviceGuard dg(ctx->device);
    efie_plan *p = new (std::nothrow) efie_plan();
    if (!p) return efie_fail(EFIE_ERR_NOMEM, "out of host memory");
    p->ctx = ctx;
    efie_status s = plan_common(p, mesh, mu, eps, patchEdge, groundEdge, V0, spreadRadius, Z0, opts);
    if (s == EFIE_OK) s = efie_geom_upload(ctx, mesh, pre, scheme, rule_order, p->g);
    // a symmetric gather writes Z(n,m) as a copy of Z(m,n): the refinement's
    // products then read only the upper triangle
    if (s == EFIE_OK) p->sw.zsym = p->g.symmetric;
    // the symmetric gather also writes the mixed solver's complex64 planes
    if (s == EFIE_OK) p->sw.planes_from_assembly = p->opts.solver == EFIE_SOLVER_MIXED && p->g.symmetric;
    if (s == EFIE_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        s = efie_fail(EFIE_ERR_CUDA, "geometry upload failed");
    if (s != EFIE_OK) {
        delete p;
        return s;
    }
    *out = p;
    return EFIE_OK;
}

extern "C" efie_status efie_plan_create_mesh(efie_ctx *ctx, const efie_mesh *mesh, const efie_precompute_opts *popts,
                                             double mu, efie_c128 eps, int32_t patchEdge, int32_t groundEdge,
                                             double V0, double spreadRadius, double Z0, const efie_sweep_opts *opts,
                                             efie_plan **out) {
    if (!ctx || !out || !popts) return efie_fail(EFIE_ERR_ARGS, "null context, options or output");
    *out = nullptr;
    EFIE_TRY(check_mesh(mesh, true));
    if (opts && opts->scheme != EFIE_SCHEME_REF)
        return efie_fail(EFIE_ERR_ARGS, "efie_plan_create_mesh builds the reference scheme's caches");
    DeviceGuard dg(ctx->device);
    efie_plan *p = new (std::nothrow) efie_plan();
    if (!p) return efie_fail(EFIE_ERR_NOMEM, "out of host memory");
    p->ctx = ctx;
    efie_status s = plan_common(p, mesh, mu, eps, patchEdge, groundEdge, V0, spreadRadius, Z0, opts);
    if (s == EFIE_OK) s = efie_geom_upload(ctx, mesh, nullptr, EFIE_SCHEME_REF, 0, p->g, popts);
    if (s == EFIE_OK) p->sw.zsym = p->g.symmetric;
    if (s == EFIE_OK) p->sw.planes_from_assembly = p->opts.solver == EFIE_SOLVER_MIXED && p->g.symmetric;
    if (s == EFIE_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        s = efie_fail(EFIE_ERR_CUDA, "geometry upload failed");
    if (s != EFIE_OK) {
        delete p;
        return s;
    }
    *out = p;
    return EFIE_OK;
}

extern "C" efie_status efie_plan_set_timing(efie_plan *p, int32_t timing) {
    if (!p) return efie_fail(EFIE_ERR_ARGS, "null plan");
    p->opts.timing = timing ? 1 : 0;
    return EFIE_OK;
}

extern "C" void efie_plan_destroy(efie_plan *p) {
    if (!p) return;
    DeviceGuard dg(p->ctx->device);
    cudaStreamSynchronize(p->ctx->stream);
    delete p;
}

// Initial guess of the frequency at sorted position q: the Lagrange
// interpolant in frequency through the (up to) three nearest solved
// neighbours, the two nearest on one side and one on the other where both
// sides have some (a quadratic through points 1-2 grid steps away), else the
// nearest one or two on the one side.
static void guess_weights(int q, const std::vector<double> &fs, const std::vector<char> &solved, GuessSpec &g,
                          int f) {
    const int Nf = (int)fs.size();
    int nodes[3], n = 0;
    int l = q - 1, r = q + 1;
    auto next_l = [&]() { while (l >= 0 && !solved[l]) l--; };
    auto next_r = [&]() { while (r < Nf && !solved[r]) r++; };
    next_l();
    next_r();
    while (n < 3 && (l >= 0 || r < Nf)) {
        const bool take_l = l >= 0 && (r >= Nf || q - l <= r - q);
        if (take_l) nodes[n++] = l--, next_l();
        else nodes[n++] = r++, next_r();
    }
    for (int t = 0; t < 3; t++) g.idx[t][f] = -1, g.w[t][f] = 0.0;
    // one-sided nodes: keep the nearest only (no extrapolation)
    bool below = false, above = false;
    for (int t = 0; t < n; t++) (nodes[t] < q ? below : above) = true;
    if (!(below && above)) n = std::min(n, 1);
    for (int t = 0; t < n; t++)
        for (int u = 0; u < t; u++)
            if (fs[nodes[t]] == fs[nodes[u]]) n = 1;   // repeated frequencies: the nearest alone
    for (int t = 0; t < n; t++) {
        double w = 1.0;
        for (int u = 0; u < n; u++)
            if (u != t) w *= (fs[q] - fs[nodes[u]]) / (fs[nodes[t]] - fs[nodes[u]]);
        g.idx[t][f] = nodes[t];
        g.w[t][f] = w;
    }
}

static bool g_warm_start_disabled = false;
extern "C" void efie_debug_disable_warm_start(int disable) { g_warm_start_disabled = disable != 0; }

extern "C" efie_status efie_plan_run(efie_plan *p, const double *freqs, int32_t Nf, efie_c128 *Zin, efie_c128 *S11,
                                     efie_c128 *I, efie_sweep_stats *st) {
    if (!p) return efie_fail(EFIE_ERR_ARGS, "null plan");
    if (Nf < 0 || (Nf > 0 && (!freqs || !Zin || !S11))) return efie_fail(EFIE_ERR_FREQS, "freqs must be double vector.");
    for (int fi = 0; fi < Nf; fi++)
        if (!(freqs[fi] > 0.0) || !std::isfinite(freqs[fi]))
            return efie_fail(EFIE_ERR_FREQS, "frequencies must be positive and finite.");
    efie_ctx *ctx = p->ctx;
    DeviceGuard dg(ctx->device);
    const int N = p->Ne;
    const size_t NN = (size_t)N * N;
    KernelLog &log = ctx->log;
    log.reset(p->opts.timing != 0);
    efie_sweep_stats local{};
    efie_sweep_stats *S = st ? st : &local;
    std::memset(S, 0, sizeof(*S));
    S->n_freq = Nf;
    EFIE_TRY(p->out.reserve(sizeof(efie_c128) * 2 * std::max(Nf, 1)));
    EFIE_TRY(p->info.reserve(sizeof(int) * std::max(Nf, 1)));
    EFIE_CUDA(cudaMemsetAsync(p->info.p, 0, sizeof(int) * std::max(Nf, 1), ctx->stream));
    const bool mixed = p->opts.solver == EFIE_SOLVER_MIXED;
    const int B = p->B;
    efie_status rc = EFIE_OK;
    // as few batches as B allows, of balanced sizes (each batch pays the
    // latency of its panel chain once).  The mixed solver with GMRES takes
    // them coarse to fine: batch b holds the frequencies at sorted positions
    // q = r_b (mod nbat), residues in van der Corput order, so every later
    // frequency starts its refinement from the interpolation of its solved
    // neighbours instead of from zero.
    const int nbat = (Nf + B - 1) / B;
    const bool warm = mixed && !p->centroid && nbat > 1 && p->opts.refine_method == EFIE_REFINE_GMRES &&
                      !g_warm_start_disabled;
    std::vector<int> ord(Nf), bstart(nbat + 1, 0), posq(Nf);   // processing index -> original, sorted position
    std::vector<double> fsorted(Nf);
    std::vector<char> solved(Nf, 0);
    {
        std::vector<int> srt(Nf);
        for (int i = 0; i < Nf; i++) srt[i] = i;
        if (warm) std::stable_sort(srt.begin(), srt.end(), [&](int a, int b) { return freqs[a] < freqs[b]; });
        for (int i = 0; i < Nf; i++) fsorted[i] = freqs[srt[i]];
        int n = 0, P = 1, bits = 0;
        while (P < nbat) P <<= 1, bits++;
        for (int i = 0, b = 0; i < (warm ? P : nbat); i++) {
            if (warm) {
                int r = 0;
                for (int t = 0; t < bits; t++) r |= ((i >> t) & 1) << (bits - 1 - t);
                if (r >= nbat) continue;
                for (int q = r; q < Nf; q += nbat) posq[n] = q, ord[n++] = srt[q];
            } else {
                const int nb = Nf / nbat + (b < Nf % nbat ? 1 : 0);
                for (int f = 0; f < nb; f++) posq[n] = n, ord[n] = srt[n], n++;
            }
            bstart[++b] = n;
        }
    }
    if (warm) EFIE_TRY(p->xall.reserve(sizeof(efie_c128) * (size_t)N * Nf));
    auto Zslot = [&](int f) -> void * { return p->Z.as<efie_c128>() + NN * f; };
    // Shared factors: with coarse-to-fine batches only the first batch of each
    // group of `group` is factored.  The frequencies of the group's other
    // batches lie between its frequencies, whose complex64 factors stay in
    // the plan's slots; each is refined with the factors of the nearest of
    // them (its assembly then leaves the planes alone).  GMRES converges to
    // the same residual target in a few more steps; a frequency that does
    // not gets the retry below, with its own factors -- which converts Z to
    // planes in every slot, so the rest of the group then factors itself.
    const int group = p->share_group;   // batches per factored batch
    const bool share = mixed && warm && group > 1 && p->sw.zsym && p->sw.sym_lu &&
                       p->opts.refine_method == EFIE_REFINE_GMRES;
    bool prev_factored = false;      // the slots hold the factors of the group's first batch
    std::vector<int> fsrc_host(p->B);
    p->sw.fsrc_on = false;
    auto set_fsrc = [&](bool identity) -> efie_status {
        p->sw.fsrc_on = !identity;
        if (identity) return EFIE_OK;
        EFIE_CUDA(cudaMemcpyAsync(p->sw.fsrc.p, fsrc_host.data(), sizeof(int) * p->B, cudaMemcpyHostToDevice,
                                  ctx->stream));
        return EFIE_OK;
    };
    for (int bi = 0; bi < nbat && rc == EFIE_OK; bi++) {
        const int f0 = bstart[bi], nb = bstart[bi + 1] - f0;
        int active[EFIE_MAX_BATCH] = {0};
        for (int f = 0; f < nb; f++) active[f] = 1;
        const bool shared = share && (bi % group) != 0 && prev_factored;
        {
            Physics ph[EFIE_MAX_BATCH];
            void *Zf[EFIE_MAX_BATCH];
            for (int f = 0; f < nb; f++) {
                ph[f] = efie_physics(freqs[ord[f0 + f]], p->mu, p->eps);
                Zf[f] = p->Z.as<efie_c128>() + NN * f;
            }
            if (p->centroid) {
                for (int f = 0; f < nb && rc == EFIE_OK; f++)
                    rc = efie_assemble_centroid_device(ctx, &p->cmesh, p->self_alpha, ph[f], Zf[f], p->scratch);
            } else {
                const PlanesOut po{p->sw.planes.as<float>(), p->sw.pstride, p->sw.ld};
                rc = efie_assemble_batch(ctx, p->g, ph, nb, Zf,
                                         p->sw.planes_from_assembly && !shared ? &po : nullptr);
            }
        }
        if (rc != EFIE_OK) break;
        bool fallback[EFIE_MAX_BATCH] = {false};
        if (mixed) {
            if (shared) {
                // each slot refines with the factors of the group's factored
                // batch's slot holding the nearest frequency
                const int gb = bi - bi % group, p0 = bstart[gb], np_ = bstart[gb + 1] - p0;
                for (int f = 0; f < p->B; f++) fsrc_host[f] = f;
                for (int f = 0; f < nb; f++) {
                    int best = 0;
                    for (int s2 = 1; s2 < np_; s2++)
                        if (std::abs(posq[p0 + s2] - posq[f0 + f]) < std::abs(posq[p0 + best] - posq[f0 + f]))
                            best = s2;
                    fsrc_host[f] = best;
                }
                rc = set_fsrc(false);
                if (rc == EFIE_OK) rc = efie_mixed_factor_prepare(ctx, p->sw, active);
                S->n_shared_factors += nb;
            } else {
                rc = set_fsrc(true);
                if (rc == EFIE_OK) rc = plan_factor(p, active, nb);
            }
            if (rc != EFIE_OK) break;
            if (!shared && bi % group == 0) prev_factored = true;
            RefineResult rr;
            const bool guess = warm && bi > 0;
            if (guess) {
                GuessSpec g;
                for (int f = 0; f < nb; f++) guess_weights(posq[f0 + f], fsorted, solved, g, f);
                rc = efie_interp_guess(ctx, N, nb, p->x.p, p->xall.p, g);
                if (rc != EFIE_OK) break;
            }
            if (p->opts.refine_method == EFIE_REFINE_CLASSICAL && p->sw.planes_from_assembly)
                for (int f = 0; f < nb && rc == EFIE_OK; f++) rc = efie_z_mirror(ctx, Zslot(f), N);
            if (rc != EFIE_OK) break;
            if (p->opts.refine_method == EFIE_REFINE_CLASSICAL)
                rc = efie_mixed_refine(ctx, p->sw, p->Z.p, NN, p->b.p, p->x.p, p->bnorm, p->opts.refine_tol,
                                       p->opts.refine_max_iter, active, &rr);
            else
                rc = efie_mixed_gmres(ctx, p->sw, p->Z.p, NN, p->b.p, p->x.p, p->bnorm, p->opts.refine_tol,
                                      p->opts.refine_max_iter, active, &rr, guess);
            if (rc != EFIE_OK) break;
            S->refine_iters_max = std::max(S->refine_iters_max, rr.iters);
            int err1[EFIE_MAX_BATCH];   // device error codes of the first attempt
            for (int f = 0; f < nb; f++) err1[f] = rr.err[f];
            if (p->sw.zsym && p->sw.sym_lu && p->opts.refine_method == EFIE_REFINE_GMRES) {
                // a frequency that missed the target with the L D L^T factors
                // is factored again as a general matrix (eager launches, from
                // Z) before the complex128 fallback
                int retry[EFIE_MAX_BATCH] = {0};
                int nr = 0;
                for (int f = 0; f < nb; f++)
                    if (!rr.converged[f] || rr.err[f]) retry[f] = 1, nr++;
                if (nr > 0) {
                    RefineResult r2;
                    const bool pfa = p->sw.planes_from_assembly;
                    // the retried frequencies refine with their own factors;
                    // the slots no longer hold the group's factors
                    rc = set_fsrc(true);
                    if (rc != EFIE_OK) break;
                    prev_factored = false;
                    // the general LU converts all of Z
                    for (int f = 0; f < nb && rc == EFIE_OK; f++)
                        if (retry[f] && pfa) rc = efie_z_mirror(ctx, Zslot(f), N);
                    if (rc != EFIE_OK) break;
                    p->sw.sym_lu = false;
                    p->sw.planes_from_assembly = false;
                    rc = efie_mixed_factor(ctx, p->sw, p->Z.p, NN, retry);
                    if (rc == EFIE_OK)
                        rc = efie_mixed_gmres(ctx, p->sw, p->Z.p, NN, p->b.p, p->x.p, p->bnorm, p->opts.refine_tol,
                                              p->opts.refine_max_iter, retry, &r2);
                    p->sw.sym_lu = true;
                    p->sw.planes_from_assembly = pfa;
                    if (rc != EFIE_OK) break;
                    S->refine_iters_max = std::max(S->refine_iters_max, r2.iters);
                    for (int f = 0; f < nb; f++)
                        if (retry[f]) rr.relres[f] = r2.relres[f], rr.converged[f] = r2.converged[f], rr.err[f] = r2.err[f];
                }
            }
            for (int f = 0; f < nb; f++) {
                // 1: zero pivot (k_diag_factor); 2, 3: a bounded wait gave up (k_trsv, k_update_tc)
                if (err1[f] == 1 || rr.err[f] == 1) S->n_zero_pivots++;
                if (err1[f] >= 2 || rr.err[f] >= 2) S->n_wait_timeouts++;
                if (!rr.converged[f] || rr.err[f]) {
                    // zero pivot, timeout or stalled refinement: complex128 LU for this frequency
                    fallback[f] = true;
                    S->n_fp64_fallback++;
                } else {
                    S->max_relres = std::max(S->max_relres, rr.relres[f]);
                }
            }
        }
        for (int f = 0; f < nb && rc == EFIE_OK; f++) {
            if (mixed && !fallback[f]) continue;
            // cuSOLVER Zgetrf/Zgetrs on all of Z: timed in class OTHER, not counted as our launches
            if (mixed && p->sw.planes_from_assembly) rc = efie_z_mirror(ctx, Zslot(f), N);
            if (rc != EFIE_OK) break;
            size_t tok = log.begin(ctx->stream);
            rc = plan_solve_fp64(p, f, f0 + f);
            if (rc == EFIE_OK) log.end(EFIE_K_OTHER, ctx->stream, tok, 8.0 / 3.0 * (double)N * N * N, 0);
        }
        if (rc != EFIE_OK) break;
        rc = efie_port_reduce(ctx, N, nb, p->x.p, p->wport.as<double>(),
                              p->centroid ? EFIE_PORT_EDGE_DIFF : p->opts.port_model, p->pe - 1, p->ge - 1, p->V0,
                              p->Z0, p->out.as<efie_c128>() + 2 * f0);
        if (rc != EFIE_OK) break;
        for (int f = 0; f < nb && rc == EFIE_OK; f++) {
            const efie_c128 *xf = p->x.as<efie_c128>() + (size_t)N * f;
            cudaError_t e = cudaSuccess;
            if (warm) {
                solved[posq[f0 + f]] = 1;
                e = cudaMemcpyAsync(p->xall.as<efie_c128>() + (size_t)N * posq[f0 + f], xf, sizeof(efie_c128) * N,
                                    cudaMemcpyDeviceToDevice, ctx->stream);
            }
            if (I && e == cudaSuccess)
                e = cudaMemcpyAsync(I + (size_t)ord[f0 + f] * N, xf, sizeof(efie_c128) * N, cudaMemcpyDeviceToHost,
                                    ctx->stream);
            if (e != cudaSuccess) rc = efie_fail(EFIE_ERR_CUDA, cudaGetErrorString(e));
        }
    }
    if (rc == EFIE_OK && Nf > 0) {
        std::vector<efie_c128> res(2 * (size_t)Nf);
        std::vector<int> info(Nf);
        cudaError_t e = cudaMemcpyAsync(res.data(), p->out.p, sizeof(efie_c128) * 2 * Nf, cudaMemcpyDeviceToHost,
                                        ctx->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(info.data(), p->info.p, sizeof(int) * Nf, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = efie_fail(EFIE_ERR_CUDA, cudaGetErrorString(e));
        else {
            for (int fi = 0; fi < Nf; fi++) {
                Zin[ord[fi]] = res[2 * fi];
                S11[ord[fi]] = res[2 * fi + 1];
            }
            int bad = -1;
            for (int fi = 0; fi < Nf; fi++)
                if (info[fi] != 0 && (bad < 0 || ord[fi] < ord[bad])) bad = fi;
            if (bad >= 0)
                rc = efie_fail(EFIE_ERR_SINGULAR, "Z is singular at frequency index " + std::to_string(ord[bad] + 1) +
                                                      " (getrf info " + std::to_string(info[bad]) + ").");
        }
    } else {
        cudaStreamSynchronize(ctx->stream);
    }
    log.resolve();
    for (int c = 0; c < EFIE_NUM_KERNEL_CLASSES; c++) {
        S->class_launches[c] = log.launches[c];
        S->class_ms[c] = log.ms[c];
        S->class_work[c] = log.work[c];
        S->n_launches += log.launches[c];
    }
    S->ms_assemble = log.ms[EFIE_K_QUAD] + log.ms[EFIE_K_NEARSELF] + log.ms[EFIE_K_GATHER];
    S->ms_factor = log.ms[EFIE_K_PANEL] + log.ms[EFIE_K_GEMM];
    S->ms_solve = log.ms[EFIE_K_TRSV] + log.ms[EFIE_K_RESIDUAL] + log.ms[EFIE_K_OTHER];
    return rc;
}

extern "C" efie_status efie_patch_sweep_fastquad(efie_ctx *ctx, const efie_mesh *mesh, const efie_prepack *pre,
                                                 const double *freqs, int32_t Nf, double mu, efie_c128 eps,
                                                 int32_t patchEdge, int32_t groundEdge, double V0, double spreadRadius,
                                                 double Z0, const efie_sweep_opts *opts, efie_c128 *Zin,
                                                 efie_c128 *S11, efie_c128 *I, efie_sweep_stats *stats) {
    efie_plan *p = nullptr;
    efie_sweep_opts o;
    if (opts) o = *opts;
    else efie_sweep_opts_default(&o);
    o.scheme = EFIE_SCHEME_REF;
    if (o.nfreq_hint <= 0) o.nfreq_hint = Nf;   // one call, one sweep: size the batches for it
    EFIE_TRY(efie_plan_create(ctx, mesh, pre, mu, eps, patchEdge, groundEdge, V0, spreadRadius, Z0, &o, 0, &p));
    efie_status s = efie_plan_run(p, freqs, Nf, Zin, S11, I, stats);
    efie_plan_destroy(p);
    return s;
}

extern "C" efie_status efie_patch_sweep_centroid(efie_ctx *ctx, const efie_mesh *mesh, const double *freqs, int32_t Nf,
                                                 double mu, efie_c128 eps, int32_t patchEdge, int32_t groundEdge,
                                                 double V0, double spreadRadius, double Z0,
                                                 const efie_sweep_opts *opts, efie_c128 *Zin, efie_c128 *S11,
                                                 efie_c128 *I, efie_sweep_stats *stats) {
    if (!ctx) return efie_fail(EFIE_ERR_ARGS, "null context");
    EFIE_TRY(check_mesh(mesh, true));
    DeviceGuard dg(ctx->device);
    efie_plan *p = new (std::nothrow) efie_plan();
    if (!p) return efie_fail(EFIE_ERR_NOMEM, "out of host memory");
    p->ctx = ctx;
    p->centroid = true;
    p->self_alpha = 0.20;  // patch_sweep_cuda.cu:269
    efie_sweep_opts o;
    if (opts) o = *opts;
    else efie_sweep_opts_default(&o);
    o.port_model = EFIE_PORT_EDGE_DIFF;
    efie_status s = plan_common(p, mesh, mu, eps, patchEdge, groundEdge, V0, spreadRadius, Z0, &o);
    if (s == EFIE_OK) {
        const int Ne = mesh->Ne, Nt = mesh->Nt, Nv = mesh->Nv;
        p->hV.assign(mesh->V, mesh->V + 3 * (size_t)Nv);
        p->hF.assign(mesh->F, mesh->F + 3 * (size_t)Nt);
        p->hpt.assign(mesh->plusTri, mesh->plusTri + Ne);
        p->hmt.assign(mesh->minusTri, mesh->minusTri + Ne);
        p->hps.assign(mesh->plusSign, mesh->plusSign + Ne);
        p->hms.assign(mesh->minusSign, mesh->minusSign + Ne);
        p->hrp.assign(mesh->rp, mesh->rp + 3 * (size_t)Ne);
        p->hrm.assign(mesh->rm, mesh->rm + 3 * (size_t)Ne);
        p->hAp.assign(mesh->Ap, mesh->Ap + Ne);
        p->hAm.assign(mesh->Am, mesh->Am + Ne);
        p->hlen.assign(mesh->len, mesh->len + Ne);
        p->cmesh = efie_mesh{Nv, Nt, Ne, p->hV.data(), p->hF.data(), nullptr, p->hpt.data(), p->hmt.data(),
                             p->hps.data(), p->hms.data(), p->hrp.data(), p->hrm.data(), p->hAp.data(),
                             p->hAm.data(), p->hlen.data()};
        // k by std::sqrt of the complex product (patch_sweep_cuda.cu:447) equals
        // the polar form used by efie_physics up to rounding.
        s = efie_plan_run(p, freqs, Nf, Zin, S11, I, stats);
    }
    efie_plan_destroy(p);
    return s;
}

// ---------------------------------------------------------------------------
// Self-test of the complex64 LU (no pivoting) used by the mixed solver.
// ---------------------------------------------------------------------------
static int g_selftest_nb = 256;
static int g_selftest_tile[3] = {256, 256, 0};   // chain tile, bulk tile, resident (1 chain, 2 bulk)
extern "C" void efie_debug_set_selftest_panel(int lu_nb) {
    g_selftest_nb = (lu_nb == 64 || lu_nb == 128 || lu_nb == 256 || lu_nb == 512) ? lu_nb : 256;
}
extern "C" void efie_debug_set_selftest_tiles(int tile_chain, int tile_bulk, int resident_chain) {
    g_selftest_tile[0] = choose_tile(tile_chain);
    g_selftest_tile[1] = choose_tile(tile_bulk);
    g_selftest_tile[2] = resident_chain & 3;
}

extern "C" efie_status efie_lu_selftest(efie_ctx *ctx, int32_t N, const efie_c128 *A, int32_t tensor_cores,
                                        efie_c128 *LU) {
    if (!ctx || N < 1 || !A || !LU) return efie_fail(EFIE_ERR_ARGS, "efie_lu_selftest: bad arguments");
    DeviceGuard dg(ctx->device);
    ctx->log.reset(false);
    SolveWork w;
    EFIE_TRY(efie_mixed_workspace(w, N, 1, g_selftest_nb));
    w.tn_chain = g_selftest_tile[0];
    w.tn_bulk = g_selftest_tile[1];
    w.resident_chain = (g_selftest_tile[2] & 1) != 0;
    w.resident_bulk = (g_selftest_tile[2] & 2) != 0;
    // a bit-exactly symmetric A takes the symmetric factorization, as a
    // sweep's Z from the symmetric gather does
    bool sym = true;
    for (int j = 0; j < N && sym; j++)
        for (int i = j + 1; i < N; i++) {
            const efie_c128 a = A[(size_t)i + (size_t)N * j], b = A[(size_t)j + (size_t)N * i];
            if (a.re != b.re || a.im != b.im) {
                sym = false;
                break;
            }
        }
    w.zsym = sym;
    DevBuf dA;
    EFIE_TRY(dA.reserve(sizeof(efie_c128) * (size_t)N * N));
    EFIE_CUDA(cudaMemcpyAsync(dA.p, A, sizeof(efie_c128) * (size_t)N * N, cudaMemcpyHostToDevice, ctx->stream));
    const int active[1] = {1};
    efie_debug_disable_tensor_cores(tensor_cores ? 0 : 1);
    efie_status s = efie_mixed_factor(ctx, w, dA.p, (size_t)N * N, active);
    efie_debug_disable_tensor_cores(0);
    EFIE_TRY(s);
    std::vector<float> pl(2 * (size_t)w.ld * N);
    EFIE_CUDA(cudaMemcpyAsync(pl.data(), w.planes.p, sizeof(float) * pl.size(), cudaMemcpyDeviceToHost, ctx->stream));
    int err = 0;
    EFIE_CUDA(cudaMemcpyAsync(&err, w.ctl.as<char>() + 36, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    EFIE_CUDA(cudaStreamSynchronize(ctx->stream));
    const float *Ar = pl.data(), *Ai = Ar + (size_t)w.ld * N;
    for (int j = 0; j < N; j++)
        for (int i = 0; i < N; i++)
            LU[(size_t)i + (size_t)N * j] = efie_c128{Ar[(size_t)i * w.ld + j], Ai[(size_t)i * w.ld + j]};
    ctx->log.resolve();
    if (err)
        return efie_fail(err == 1 ? EFIE_ERR_SINGULAR : EFIE_ERR_TIMEOUT,
                         "LU self-test: device error flag " + std::to_string(err));
    return EFIE_OK;
}
