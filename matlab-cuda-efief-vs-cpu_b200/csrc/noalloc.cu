// Centroid assembly (gassemble) that allocates no device memory.
//
// Some callers cannot call cudaMalloc: processes that must stay inside a
// device-memory budget fixed at start-up (an allocation later could fail or
// evict another tenant's memory), or hosts (a MATLAB gpuArray workflow, a
// real-time loop) that own every device buffer themselves and do not let a
// library allocate behind their back.  efie_gassemble_zv_noalloc serves them:
// the caller passes every input and output as a device pointer, and the
// scratch the kernels need (per-edge side data, per-triangle softening
// lengths, a status word) lives in one file-scope __device__ array of fixed
// size that every GPU loading this library keeps until the process exits.
//
// Limits: Ne <= EFIE_NOALLOC_MAX_NE and Nt <= EFIE_NOALLOC_MAX_NT.  All calls
// on a device share the array, so calls that overlap on the GPU (different
// streams, or host threads) race; serialise them.  The first call on a
// device looks up the array's device address (cudaGetSymbolAddress with that
// device current) and keeps it for the life of the process; make that first
// call before any stream capture, and do not use this entry point across a
// cudaDeviceReset of that device (the kept address belongs to the destroyed
// context).  Each call reads its status word back and synchronises `stream`
// before it returns.
#include <cmath>
#include <cstring>
#include <mutex>

#include "efie_internal.h"

namespace {

constexpr int kMaxNe = EFIE_NOALLOC_MAX_NE;
constexpr int kMaxNt = EFIE_NOALLOC_MAX_NT;
constexpr double kPi = 3.141592653589793238462643383279502884;

// One edge side (plus or minus triangle) at its triangle's centroid.
struct NaSide {
    double px, py, pz, fx, fy, fz, div, w, t, pad;
};

// Layout of the scratch array (in doubles): side data, softening, status.
constexpr size_t kSideDoubles = sizeof(NaSide) / sizeof(double) * 2 * (size_t)kMaxNe;
constexpr size_t kScratchDoubles = kSideDoubles + (size_t)kMaxNt * 4 + 8;

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

std::mutex g_mutex;
void *g_scratch_ptr[64] = {nullptr};

// status bits
constexpr int kBadF = 1, kBadTri = 2, kBadE = 4, kNoWeights = 8;

// per triangle: centroid and self softening a = selfAlpha * sqrt(A / pi)
// (gassemble_ZV_EFIE_RWG_DIFF_GPU_FAST.cu:224-247)
__global__ void k_na_triangles(int Nv, int Nt, const double *__restrict__ V, const int *__restrict__ F,
                               double selfAlpha, double *__restrict__ tri, int *__restrict__ status) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= Nt) return;
    int id[3];
    for (int j = 0; j < 3; j++) {
        id[j] = F[t + (size_t)j * Nt] - 1;
        if (id[j] < 0 || id[j] >= Nv) {
            atomicOr(status, kBadF);
            return;
        }
    }
    double r[3][3];
    for (int j = 0; j < 3; j++)
        for (int c = 0; c < 3; c++) r[j][c] = V[id[j] + (size_t)c * Nv];
    for (int c = 0; c < 3; c++) tri[4 * t + c] = (r[0][c] + r[1][c] + r[2][c]) / 3.0;
    const double e1x = r[1][0] - r[0][0], e1y = r[1][1] - r[0][1], e1z = r[1][2] - r[0][2];
    const double e2x = r[2][0] - r[0][0], e2y = r[2][1] - r[0][1], e2z = r[2][2] - r[0][2];
    const double cx = e1y * e2z - e1z * e2y, cy = e1z * e2x - e1x * e2z, cz = e1x * e2y - e1y * e2x;
    const double A = 0.5 * sqrt(cx * cx + cy * cy + cz * cz);
    tri[4 * t + 3] = selfAlpha * sqrt(A / kPi);
}

// per edge side: position, basis value and divergence at the centroid, weight = area
// (gassemble_ZV_EFIE_RWG_DIFF_GPU_FAST.cu:261-299)
__global__ void k_na_sides(int Nt, int Ne, const int *__restrict__ plusTri, const int *__restrict__ minusTri,
                           const int *__restrict__ plusSign, const int *__restrict__ minusSign,
                           const double *__restrict__ rp, const double *__restrict__ rm, const double *__restrict__ Ap,
                           const double *__restrict__ Am, const double *__restrict__ len,
                           const double *__restrict__ tri, NaSide *__restrict__ side, int *__restrict__ status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 2 * Ne) return;
    const int e = i >> 1, sd = i & 1;
    NaSide o;
    memset(&o, 0, sizeof(o));
    const int t = sd == 0 ? plusTri[e] : minusTri[e];
    if (t < 0 || t > Nt) {
        atomicOr(status, kBadTri);
        side[i] = o;
        return;
    }
    const double A = sd == 0 ? Ap[e] : Am[e];
    o.t = t;
    o.w = t > 0 ? A : 0.0;
    if (t > 0) {
        o.px = tri[4 * (t - 1)];
        o.py = tri[4 * (t - 1) + 1];
        o.pz = tri[4 * (t - 1) + 2];
    }
    if (t > 0 && A > 0) {
        const double l = len[e];
        const int sg = sd == 0 ? plusSign[e] : minusSign[e];
        const double sc = (double)sg * (l / (2.0 * A));
        const double *v = sd == 0 ? rp : rm;
        const double vx = v[e], vy = v[e + Ne], vz = v[e + 2 * (size_t)Ne];
        if (sd == 0) {
            o.fx = sc * (o.px - vx); o.fy = sc * (o.py - vy); o.fz = sc * (o.pz - vz);
            o.div = (double)sg * (l / A);
        } else {
            o.fx = sc * (vx - o.px); o.fy = sc * (vy - o.py); o.fz = sc * (vz - o.pz);
            o.div = (double)sg * (-(l / A));
        }
    }
    side[i] = o;
}

__device__ __forceinline__ double block_sum(double v, double *sh) {
    const int tid = threadIdx.x;
    sh[tid] = v;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (tid < o) sh[tid] += sh[tid + o];
        __syncthreads();
    }
    const double r = sh[0];
    __syncthreads();
    return r;
}

__device__ __forceinline__ double block_minmax(double v, double *sh, bool mx) {
    const int tid = threadIdx.x;
    sh[tid] = v;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (tid < o) sh[tid] = mx ? fmax(sh[tid], sh[tid + o]) : fmin(sh[tid], sh[tid + o]);
        __syncthreads();
    }
    const double r = sh[0];
    __syncthreads();
    return r;
}

// Vrhs = +V0/2 wPatch - V0/2 wGnd, normalised Gaussian weights of edge-centre
// distance on the port edge's layer (ggassemble_ZV_EFIE_RWG_DIFF_GPU_FAST.cu:492-540).
// One CTA of 1024 threads; the weights are recomputed instead of stored.
__global__ void __launch_bounds__(1024) k_na_rhs(int Nv, int Ne, const double *__restrict__ V,
                                                 const int *__restrict__ E, int pe, int ge, double V0, double spread,
                                                 double2 *__restrict__ Vrhs, int *__restrict__ status) {
    __shared__ double sh[1024];
    const int tid = threadIdx.x;
    auto centre = [&](int e, double &x, double &y, double &z) -> bool {
        const int a = E[e] - 1, b = E[e + Ne] - 1;
        if (a < 0 || a >= Nv || b < 0 || b >= Nv) return false;
        x = 0.5 * (V[a] + V[b]);
        y = 0.5 * (V[a + Nv] + V[b + Nv]);
        z = 0.5 * (V[a + 2 * (size_t)Nv] + V[b + 2 * (size_t)Nv]);
        return true;
    };
    double zmin = 1e100, zmax = -1e100;
    int bad = 0;
    for (int e = tid; e < Ne; e += 1024) {
        double x, y, z;
        if (!centre(e, x, y, z)) { bad = 1; continue; }
        zmin = fmin(zmin, z);
        zmax = fmax(zmax, z);
    }
    if (bad) atomicOr(status, kBadE);
    zmin = block_minmax(zmin, sh, false);
    zmax = block_minmax(zmax, sh, true);
    if (*((volatile int *)status) & kBadE) return;
    const double zmid = 0.5 * (zmin + zmax);
    double px, py, pz, gx, gy, gz;
    centre(pe, px, py, pz);
    centre(ge, gx, gy, gz);
    const int lp = pz > zmid ? 1 : -1, lg = gz > zmid ? 1 : -1;
    auto weight = [&](int e, double ox, double oy, double oz, int layer0) -> double {
        double x, y, z;
        centre(e, x, y, z);
        if ((z > zmid ? 1 : -1) != layer0) return 0.0;
        const double dx = x - ox, dy = y - oy, dz = z - oz;
        const double dist = sqrt(dx * dx + dy * dy + dz * dz);
        return exp(-(dist / spread) * (dist / spread));
    };
    double sp = 0.0, sg = 0.0;
    for (int e = tid; e < Ne; e += 1024) {
        sp += weight(e, px, py, pz, lp);
        sg += weight(e, gx, gy, gz, lg);
    }
    sp = block_sum(sp, sh);
    sg = block_sum(sg, sh);
    if (!(sp >= 1e-30) || !(sg >= 1e-30)) {
        if (tid == 0) atomicOr(status, kNoWeights);
        return;
    }
    for (int e = tid; e < Ne; e += 1024) {
        const double v = (+V0 / 2.0) * (weight(e, px, py, pz, lp) / sp) + (-V0 / 2.0) * (weight(e, gx, gy, gz, lg) / sg);
        Vrhs[e] = make_double2(v, 0.0);
    }
}

__device__ __forceinline__ void green(double kr, double ki, double R, double &gr, double &gi) {
    double s, c;
    sincos(kr * R, &s, &c);
    double inv = 1.0 / (4.0 * kPi * R);
    if (ki != 0.0) inv *= exp(ki * R);
    gr = c * inv;
    gi = -s * inv;
}

// kernel_Z_centroid (gassemble_ZV_EFIE_RWG_DIFF_GPU_FAST.cu:49-106) over the side data
__global__ void __launch_bounds__(256) k_na_centroid_z(int Ne, const NaSide *__restrict__ side,
                                                       const double *__restrict__ tri, double kr, double ki,
                                                       double alr, double ali, double ber, double bei,
                                                       double2 *__restrict__ Z, const int *__restrict__ status) {
    if (*status) return;
    const int m = blockIdx.x * 64 + (threadIdx.x & 63);
    const int n = blockIdx.y * 4 + (threadIdx.x >> 6);
    if (m >= Ne || n >= Ne) return;
    double zr = 0.0, zi = 0.0;
    for (int sa = 0; sa < 2; sa++) {
        const NaSide A = side[2 * m + sa];
        if (A.w == 0.0 || A.t == 0.0) continue;
        for (int sb = 0; sb < 2; sb++) {
            const NaSide B = side[2 * n + sb];
            if (B.w == 0.0 || B.t == 0.0) continue;
            const double dx = A.px - B.px, dy = A.py - B.py, dz = A.pz - B.pz;
            double R = sqrt(dx * dx + dy * dy + dz * dz);
            if (A.t == B.t) {
                const double a = tri[4 * ((int)A.t - 1) + 3];
                R = sqrt(R * R + a * a);
            }
            R = fmax(R, 1e-15);
            double gr, gi;
            green(kr, ki, R, gr, gi);
            const double ff = A.fx * B.fx + A.fy * B.fy + A.fz * B.fz;
            const double dv = A.div * B.div;
            const double w = A.w * B.w;
            const double vr = gr * (ff * w), vi = gi * (ff * w);
            const double sr = gr * (dv * w), si = gi * (dv * w);
            zr += (alr * vr - ali * vi) + (ber * sr - bei * si);
            zi += (alr * vi + ali * vr) + (ber * si + bei * sr);
        }
    }
    Z[(size_t)m + (size_t)Ne * n] = make_double2(zr, zi);
}

// Device address of the scratch array on `device` (looked up once per device).
efie_status scratch_on(int device, double **out) {
    if (device < 0 || device >= 64) return efie_fail(EFIE_ERR_ARGS, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_ptr[device]) {
        int prev = -1;
        EFIE_CUDA(cudaGetDevice(&prev));
        if (prev != device) EFIE_CUDA(cudaSetDevice(device));
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (prev != device) cudaSetDevice(prev);
        if (e != cudaSuccess)
            return efie_fail(EFIE_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_scratch_ptr[device] = p;
    }
    *out = static_cast<double *>(g_scratch_ptr[device]);
    return EFIE_OK;
}

}  // namespace

extern "C" efie_status efie_gassemble_zv_noalloc(int device, void *stream, int32_t Nv, int32_t Nt, int32_t Ne,
                                                 const double *V, const int32_t *F, const int32_t *E,
                                                 const int32_t *plusTri, const int32_t *minusTri,
                                                 const int32_t *plusSign, const int32_t *minusSign,
                                                 const double *rp, const double *rm, const double *Ap,
                                                 const double *Am, const double *len, efie_c128 k, double omega,
                                                 double mu, efie_c128 eps, const double exc[5], efie_c128 *Z,
                                                 efie_c128 *Vrhs) {
    if (Ne > kMaxNe || Nt > kMaxNt)
        return efie_fail(EFIE_ERR_ARGS, "efie_gassemble_zv_noalloc: Ne must be <= " + std::to_string(kMaxNe) +
                                            " and Nt <= " + std::to_string(kMaxNt) + " (got Ne=" +
                                            std::to_string(Ne) + ", Nt=" + std::to_string(Nt) + ")");
    if (Nv < 1 || !V) return efie_fail(EFIE_ERR_V, "V must be [Nv x 3] double.");
    if (Nt < 1 || !F) return efie_fail(EFIE_ERR_F, "F must be [Nt x 3] int32.");
    if (Ne < 1 || !E) return efie_fail(EFIE_ERR_E, "E must be [Ne x 2] int32.");
    if (!plusTri || !minusTri || !plusSign || !minusSign || !rp || !rm || !Ap || !Am || !len)
        return efie_fail(EFIE_ERR_RWG, "missing RWG arrays.");
    if (!exc)
        return efie_fail(EFIE_ERR_EXC,
                         "exc must be double vector len>=5: [patchEdge, groundEdge, V0, spreadRadius, selfAlpha].");
    const int pe = (int)exc[0], ge = (int)exc[1];
    if (!(pe >= 1 && pe <= Ne)) return efie_fail(EFIE_ERR_PORT, "patchEdge out of range.");
    if (!(ge >= 1 && ge <= Ne)) return efie_fail(EFIE_ERR_PORT, "groundEdge out of range.");
    if (!Z || !Vrhs) return efie_fail(EFIE_ERR_ARGS, "null output");
    double *scratch = nullptr;
    EFIE_TRY(scratch_on(device, &scratch));
    int prev = -1;
    EFIE_CUDA(cudaGetDevice(&prev));
    if (prev != device) EFIE_CUDA(cudaSetDevice(device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    NaSide *side = reinterpret_cast<NaSide *>(scratch);
    double *tri = scratch + kSideDoubles;
    int *status = reinterpret_cast<int *>(tri + (size_t)kMaxNt * 4);
    const Physics ph = efie_physics_k(k, omega, mu, eps);
    efie_status rc = EFIE_OK;
    int hstatus = 0;
    cudaError_t e = cudaMemsetAsync(status, 0, sizeof(int), s);  // the status word starts at zero every call
    if (e == cudaSuccess) {
        k_na_triangles<<<(Nt + 255) / 256, 256, 0, s>>>(Nv, Nt, V, F, exc[4], tri, status);
        k_na_sides<<<(2 * Ne + 255) / 256, 256, 0, s>>>(Nt, Ne, plusTri, minusTri, plusSign, minusSign, rp, rm, Ap,
                                                        Am, len, tri, side, status);
        k_na_rhs<<<1, 1024, 0, s>>>(Nv, Ne, V, E, pe - 1, ge - 1, exc[2], exc[3], reinterpret_cast<double2 *>(Vrhs),
                                    status);
        dim3 gg((Ne + 63) / 64, (Ne + 3) / 4);
        k_na_centroid_z<<<gg, 256, 0, s>>>(Ne, side, tri, ph.kr, ph.ki, ph.alr, ph.ali, ph.ber, ph.bei,
                                           reinterpret_cast<double2 *>(Z), status);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hstatus, status, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) rc = efie_fail(EFIE_ERR_CUDA, std::string("efie_gassemble_zv_noalloc: ") + cudaGetErrorString(e));
    else if (hstatus & kBadF) rc = efie_fail(EFIE_ERR_F, "F has invalid indices.");
    else if (hstatus & kBadTri) rc = efie_fail(EFIE_ERR_RWG, "plusTri/minusTri out of range.");
    else if (hstatus & kBadE) rc = efie_fail(EFIE_ERR_E, "E has invalid indices.");
    else if (hstatus & kNoWeights) rc = efie_fail(EFIE_ERR_RHS, "spreadRadius too small (no weights).");
    if (prev != device) cudaSetDevice(prev);
    return rc;
}
