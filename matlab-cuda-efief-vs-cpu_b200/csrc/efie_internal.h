// Internal declarations shared by the native sources of libefie_b200.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>

#include "../../include/efie_b200.h"

// Record `msg` as the calling thread's last error and return `s`.
efie_status efie_fail(efie_status s, const std::string &msg);

// tri_quad_rule points/weights (u, v, w arrays of at least 7 entries).
int efie_quad_rule(int order, double *u, double *v, double *w);

#ifdef __CUDACC__
#include <cuda_runtime.h>
#include <cusolverDn.h>

#define EFIE_CUDA(call)                                                                      \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return efie_fail(EFIE_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

#define EFIE_TRY(call)                         \
    do {                                       \
        efie_status s_ = (call);               \
        if (s_ != EFIE_OK) return s_;          \
    } while (0)

inline efie_status efie_cuda_check(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return EFIE_OK;
    return efie_fail(EFIE_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// Makes `dev` current for the lifetime of the guard.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

// Device memory of the current device through a per-device cache: a freed
// block is kept (after the device has finished with it, like cudaFree) and
// handed to a later request of at most twice its size, so a caller that
// creates and destroys plans of the same problem repeatedly stops paying for
// cudaMalloc/cudaFree of gigabytes.  The cache is capped (40 % of the device)
// and emptied by efie_pool_trim (context destruction) or when cudaMalloc fails.
void *efie_pool_get(size_t n, size_t *got, cudaError_t *err);
void efie_pool_put(void *p, size_t bytes);
void efie_pool_trim(int device);
size_t efie_pool_cached(int device);

// A device allocation owned by a context or plan; grows, never shrinks.
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    efie_status reserve(size_t n) {
        if (n <= bytes) return EFIE_OK;
        release();
        cudaError_t e = cudaSuccess;
        size_t got = 0;
        p = efie_pool_get(n ? n : 1, &got, &e);
        if (!p) return efie_fail(EFIE_ERR_NOMEM, std::string("cudaMalloc failed: ") + cudaGetErrorString(e));
        bytes = got;
        return EFIE_OK;
    }
    void release() {
        if (p) efie_pool_put(p, bytes);
        p = nullptr;
        bytes = 0;
    }
    template <class T> T *as() const { return static_cast<T *>(p); }
    ~DevBuf() { release(); }
};

#include <vector>

// Per-launch accounting: every launch is counted per kernel class; with
// timing on, a pair of CUDA events brackets it on the launching stream and
// the durations are resolved once, after the sweep's final synchronisation.
struct KernelLog {
    bool timing = false;
    int launches[EFIE_NUM_KERNEL_CLASSES] = {0};
    double work[EFIE_NUM_KERNEL_CLASSES] = {0};
    double ms[EFIE_NUM_KERNEL_CLASSES] = {0};
    struct Ent { int cls; size_t a, b; };
    std::vector<cudaEvent_t> pool;
    std::vector<Ent> ents;
    size_t used = 0;
    cudaEvent_t next() {
        if (used == pool.size()) {
            cudaEvent_t e = nullptr;
            cudaEventCreate(&e);
            pool.push_back(e);
        }
        return pool[used++];
    }
    // Call before a launch; returns a token for end().
    size_t begin(cudaStream_t s) {
        if (!timing) return 0;
        size_t i = used;
        cudaEventRecord(next(), s);
        return i;
    }
    void end(int cls, cudaStream_t s, size_t tok, double w, int nlaunch = 1) {
        launches[cls] += nlaunch;
        work[cls] += w;
        if (!timing) return;
        size_t i = used;
        cudaEventRecord(next(), s);
        ents.push_back(Ent{cls, tok, i});
    }
    void reset(bool t) {
        timing = t;
        for (int c = 0; c < EFIE_NUM_KERNEL_CLASSES; c++) launches[c] = 0, work[c] = 0, ms[c] = 0;
        ents.clear();
        used = 0;
    }
    // After the stream has been synchronised.
    void resolve() {
        for (const Ent &e : ents) {
            float t = 0.f;
            if (cudaEventElapsedTime(&t, pool[e.a], pool[e.b]) == cudaSuccess) ms[e.cls] += t;
        }
        ents.clear();
        used = 0;
    }
    ~KernelLog() {
        for (cudaEvent_t e : pool) cudaEventDestroy(e);
    }
};

struct efie_ctx {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    cusolverDnHandle_t solver = nullptr;
    int num_sms = 0;
    int cc_major = 0;
    DevBuf status;   // device-side error flags of bounded waits (int32[8])
    KernelLog log;
};

// Device geometry of one sweep/assembly problem (uploaded once per plan).
struct GeomDev {
    int Ne = 0, Nt = 0, Nq = 0, Nq2 = 0, NsS = 0, NsN = 0;
    int n_near = 0;           // number of near (t1 < t2) pairs
    bool symmetric = true;    // nearMat symmetric -> regular moments only for t1 <= t2
    int scheme = EFIE_SCHEME_REF;
    double near_alpha = 0.0;
    DevBuf origin;            // double4[Nt]  (origin of local coordinates)
    DevBuf reg_pts;           // double4[Nt*Nq]  (rho - relative to origin, w)
    DevBuf near_pts;          // double4[Nt*NsN*Nq2]
    DevBuf self_pts;          // double4[Nt*NsS*Nq2]
    DevBuf self_a;            // double[Nt*NsS]
    DevBuf aeq;               // double[Nt]
    DevBuf near_mask;         // uint8[Nt*Nt] (1 = near or self: not a regular pair)
    DevBuf near_list;         // int2[n_near] (t1 < t2)
    DevBuf edge_tri;          // int32[2*Ne] (side 0 = plus, 1 = minus; -1 = none)
    DevBuf edge_cd;           // double4[2*Ne] (delta = free vertex - origin, c)
    DevBuf tri_vtx;           // double4[3*Nt] vertices relative to origin (extraction scheme)
    DevBuf adj_list;          // int2[] vertex-adjacent pairs t1 < t2 (extraction scheme)
    int n_adj = 0;
    DevBuf moments;           // double2[9 or 8][npairs]: component-major pair values (assemble.cu)
    size_t npairs = 0;
    bool combo = false;       // edge-combination form (9 values per pair) in use
    int mf = 1;               // frequencies whose pair values fit the moment buffer together
    DevBuf tri_d;             // double4[3*Nt] free-vertex vectors per triangle slot
    DevBuf edge_tl;           // int32[2*Ne] 4 t + slot per RWG side (-1 = none)
    DevBuf edge_c;            // double[2*Ne] RWG coefficient c per side
    DevBuf reg_tiles;         // int2[n_reg_tiles] (t1 block, t2 block) of the symmetric regular-pair launches
    int n_reg_tiles = 0;
};

// Per-frequency physics: k = w sqrt(mu eps) (principal branch), alpha = j w mu,
// beta = 1/(j w eps)  (patch_sweep_fastquad_cuda.cu:713-743).
struct Physics {
    double kr, ki, alr, ali, ber, bei;
};
Physics efie_physics(double freq, double mu, efie_c128 eps);
Physics efie_physics_k(efie_c128 k, double omega, double mu, efie_c128 eps);

// assemble.cu
// pre == nullptr with the reference scheme: the caches and the near-pair
// list are computed on the device from V/F with the options `popts`
efie_status efie_geom_upload(efie_ctx *ctx, const efie_mesh *mesh, const efie_prepack *pre, int scheme,
                             int rule_order, GeomDev &g, const efie_precompute_opts *popts = nullptr);
// The batch assembly with complex64 planes writes Z's upper triangle (and
// its 128 x 128 diagonal blocks): this completes the lower triangle of one
// slot for the paths that read all of Z (complex128 fallback, general-LU
// retry, classical refinement)
efie_status efie_z_mirror(efie_ctx *ctx, void *Z, int Ne);
// precompute.cu: efie_precompute + efie_precompute_pack on the device, straight
// into the plan's layout (origins, cache points, near-pair list)
efie_status efie_geom_precompute_device(efie_ctx *ctx, const efie_mesh *mesh, const efie_precompute_opts *o,
                                        GeomDev &g);
// pr (optional, symmetric gather only): also write the complex64 working
// matrix of the mixed solver as FP32 planes, re at pr[m * ld + n], im at
// pr[(Ne + m) * ld + n]
efie_status efie_assemble_device(efie_ctx *ctx, GeomDev &g, const Physics &ph, void *Z /*c128 Ne*Ne*/,
                                 float *pr = nullptr, int ld = 0);
// the planes of frequency slot f at p + pstride * f
struct PlanesOut {
    float *p;
    size_t pstride;
    int ld;
};
// nf frequencies of a batch into Z[0 .. nf-1] (equally spaced runs share the
// regular-pair evaluation), and into the planes of slots 0 .. nf-1 when po is set
efie_status efie_assemble_batch(efie_ctx *ctx, GeomDev &g, const Physics *ph, int nf, void *const *Z,
                                const PlanesOut *po = nullptr);
efie_status efie_assemble_centroid_device(efie_ctx *ctx, const efie_mesh *mesh, double selfAlpha,
                                          const Physics &ph, void *Z, DevBuf &scratch);
#endif
