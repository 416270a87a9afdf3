// Flexible GMRES with the complex64 LU as right preconditioner, batched over
// the frequencies of a solve batch.
//
// Classical refinement (x += U^-1 L^-1 r) contracts the error by about
// u32 * cond(Z) per step; where that product approaches 1 -- frequencies near
// a resonance of the structure -- it stalls.  GMRES on Z M^-1 u = b instead
// minimises the true residual over the Krylov space, so a few outlying
// eigenvalues of Z M^-1 cost a few extra steps rather than convergence.
//
//   r0 = b - Z x0,  beta = ||r0||,  v0 = r0 / beta,  g = beta e0
//   for j = 0, 1, ...:
//       z_j = M^-1 v_j          complex64 triangular solves, stored complex128
//       w   = Z z_j             complex128 GEMV over the column-major Z
//       h   = V^H w; w -= V h   twice (classical Gram-Schmidt with
//                               re-orthogonalisation), h_{j+1,j} = ||w||
//       v_{j+1} = w / h_{j+1,j}
//       complex Givens rotations reduce H to upper triangular R; |g_{j+1}|
//       is the residual norm of x0 + Zm y
//   y = R^-1 g,  x = x0 + Zm y,  then the true residual decides convergence
//   (a cycle that did not reach the tolerance restarts from x).
// Storing z_j (flexible GMRES) makes Z Zm = V H hold to complex128 rounding
// whatever the preconditioner's precision, so the residual estimate is the
// complex128 one.
//
// Every kernel carries the frequency in its grid and returns at once for a
// frequency whose cycle has stopped; the host polls the stop flags after
// every step from the third on.  Per-frequency state lives in GmState (device memory).
#include <algorithm>
#include <cmath>
#include <vector>

#include "efie_internal.h"
#include "solve.h"
#include "tma.h"

namespace {

constexpr int GM_M = 32;      // Arnoldi steps per cycle (restart length)
constexpr int ROWS = 256;     // rows per CTA of the orthogonalisation kernels

struct GmState {
    int j;            // Arnoldi steps done in this cycle
    int stop;         // the cycle has finished for this frequency
    int pad0, pad1;
    double beta;      // norm of the cycle's starting residual
    double inv_h;     // 1 / h_{j+1,j} of the last step (0 on breakdown)
    double res;       // |g_{j+1}|: residual norm of the current iterate
    double tolabs;    // stop when res <= tolabs
    double2 H[(GM_M + 1) * GM_M];   // column-major, leading dimension GM_M + 1
    double cs[GM_M];
    double2 sn[GM_M];
    double2 g[GM_M + 1];
    double2 y[GM_M];
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {  // conj(a) * b
    return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

__device__ __forceinline__ int *ctl_conv(char *ctl, int f) { return reinterpret_cast<int *>(ctl + 64 * f + 28); }
__device__ __forceinline__ int *ctl_skip(char *ctl, int f) { return reinterpret_cast<int *>(ctl + 64 * f + 32); }

// Cycle start: v0 = r / ||r|| (r at V slot 0 from the residual kernel), its
// complex64 copy for the preconditioner, and the frequency's Arnoldi state.
__global__ void __launch_bounds__(256) k_gm_start(int N, int B, double2 *__restrict__ V, float2 *__restrict__ rfb,
                                                  int vstride, GmState *__restrict__ st, char *__restrict__ ctl,
                                                  double tol_inner, const int *__restrict__ active) {
    const int f = blockIdx.y;
    const int conv = *ctl_conv(ctl, f) || !active[f];   // empty slots count as converged
    const double *red = reinterpret_cast<const double *>(ctl + 64 * f);
    const double beta = red[2] * red[1];   // rel * ||b||
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        GmState &s = st[f];
        s.j = 0;
        s.stop = conv || !(beta > 0.0);
        s.beta = beta;
        s.res = beta;
        s.inv_h = 0.0;
        s.tolabs = tol_inner * red[1];
        s.g[0] = make_double2(beta, 0.0);
        for (int i = 1; i <= GM_M; i++) s.g[i] = make_double2(0.0, 0.0);
        *ctl_skip(ctl, f) = s.stop;
    }
    if (conv || !(beta > 0.0)) return;
    const int n = blockIdx.x * 256 + threadIdx.x;
    if (n >= N) return;
    const double inv = 1.0 / beta;
    double2 *v = V + (size_t)N * f;
    const double2 r = v[n];
    const double2 q = make_double2(r.x * inv, r.y * inv);
    v[n] = q;
    rfb[(size_t)vstride * f + n] = make_float2((float)q.x, (float)q.y);
}

// w_f = Z_f z_f (complex128 GEMV, column-major Z): 32 rows x 8 column groups
// per CTA, grid (rows / 32, B).
__global__ void __launch_bounds__(256) k_gm_matvec(int N, const double2 *__restrict__ Zb, size_t zstride,
                                                   const double2 *__restrict__ zb, double2 *__restrict__ wb,
                                                   const GmState *__restrict__ st) {
    const int f = blockIdx.y;
    if (st[f].stop) return;
    const double2 *Z = Zb + zstride * f;
    const double2 *z = zb + (size_t)N * f;
    __shared__ double2 part[8][32];
    const int lane = threadIdx.x & 31, g = threadIdx.x >> 5;
    const int m = blockIdx.x * 32 + lane;
    double2 s = make_double2(0.0, 0.0);
    if (m < N) {
        for (int n = g; n < N; n += 8) {
            const double2 a = Z[(size_t)m + (size_t)N * n];
            const double2 v = z[n];
            s.x += a.x * v.x - a.y * v.y;
            s.y += a.x * v.y + a.y * v.x;
        }
    }
    part[g][lane] = s;
    __syncthreads();
    if (g == 0 && m < N) {
        double2 t = make_double2(0.0, 0.0);
        for (int i = 0; i < 8; i++) {
            t.x += part[i][lane].x;
            t.y += part[i][lane].y;
        }
        wb[(size_t)N * f + m] = t;
    }
}

// Partial sums of h_i = v_i^H w (i < nv) over this CTA's rows:
// part[(f * nch + chunk) * (GM_M + 1) + i].
__global__ void __launch_bounds__(ROWS) k_gm_dot(int N, int B, int nv, const double2 *__restrict__ V,
                                                 const double2 *__restrict__ wb, double2 *__restrict__ part,
                                                 const GmState *__restrict__ st) {
    const int f = blockIdx.y;
    if (st[f].stop) return;
    __shared__ double2 sm[GM_M + 1][ROWS / 32];
    const int n = blockIdx.x * ROWS + threadIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const double2 w = n < N ? wb[(size_t)N * f + n] : make_double2(0.0, 0.0);
    for (int i = 0; i < nv; i++) {
        double2 p = make_double2(0.0, 0.0);
        if (n < N) p = cmulc(V[((size_t)i * B + f) * N + n], w);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            p.x += __shfl_xor_sync(0xffffffffu, p.x, o);
            p.y += __shfl_xor_sync(0xffffffffu, p.y, o);
        }
        if (lane == 0) sm[i][warp] = p;
    }
    __syncthreads();
    if (threadIdx.x < nv) {
        double2 t = make_double2(0.0, 0.0);
        for (int q = 0; q < ROWS / 32; q++) {
            t.x += sm[threadIdx.x][q].x;
            t.y += sm[threadIdx.x][q].y;
        }
        part[((size_t)f * gridDim.x + blockIdx.x) * (GM_M + 1) + threadIdx.x] = t;
    }
}

// h = sum of the partials; w -= V h on this CTA's rows; CTA 0 adds h to
// column j of H.  With norm_part, also the partial sums of |w|^2 after the
// update: norm_part[f * nch + chunk].
__global__ void __launch_bounds__(ROWS) k_gm_axpy(int N, int B, int nv, int j, const double2 *__restrict__ V,
                                                  double2 *__restrict__ wb, const double2 *__restrict__ part,
                                                  GmState *__restrict__ st, double *__restrict__ norm_part) {
    const int f = blockIdx.y;
    if (st[f].stop) return;
    __shared__ double2 h[GM_M + 1];
    __shared__ double sq[ROWS / 32];
    const int nch = gridDim.x;
    if (threadIdx.x < nv) {
        double2 t = make_double2(0.0, 0.0);
        const double2 *p = part + (size_t)f * nch * (GM_M + 1) + threadIdx.x;
        for (int c = 0; c < nch; c++) {
            t.x += p[(size_t)c * (GM_M + 1)].x;
            t.y += p[(size_t)c * (GM_M + 1)].y;
        }
        h[threadIdx.x] = t;
        if (blockIdx.x == 0) {
            double2 &H = st[f].H[threadIdx.x + (GM_M + 1) * j];
            H.x += t.x;
            H.y += t.y;
        }
    }
    __syncthreads();
    const int n = blockIdx.x * ROWS + threadIdx.x;
    double q = 0.0;
    if (n < N) {
        double2 w = wb[(size_t)N * f + n];
        for (int i = 0; i < nv; i++) {
            const double2 v = V[((size_t)i * B + f) * N + n];
            const double2 hv = cmul(h[i], v);
            w.x -= hv.x;
            w.y -= hv.y;
        }
        wb[(size_t)N * f + n] = w;
        q = w.x * w.x + w.y * w.y;
    }
    if (norm_part) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) q += __shfl_xor_sync(0xffffffffu, q, o);
        if ((threadIdx.x & 31) == 0) sq[threadIdx.x >> 5] = q;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int i = 0; i < ROWS / 32; i++) t += sq[i];
            norm_part[(size_t)f * nch + blockIdx.x] = t;
        }
    }
}

// Zero column j of H before the two Gram-Schmidt passes add into it.
__global__ void k_gm_zero_col(int B, int j, GmState *__restrict__ st) {
    const int f = blockIdx.x, i = threadIdx.x;
    if (st[f].stop || i > GM_M) return;
    st[f].H[i + (GM_M + 1) * j] = make_double2(0.0, 0.0);
}

// One thread per frequency: h_{j+1,j} = ||w||, Givens rotations, residual
// estimate and the stop decision.
__global__ void k_gm_arnoldi(int B, int j, int nch, const double *__restrict__ norm_part, GmState *__restrict__ st,
                             char *__restrict__ ctl) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= B) return;
    GmState &s = st[f];
    if (s.stop) return;
    double nn = 0.0;
    for (int c = 0; c < nch; c++) nn += norm_part[(size_t)f * nch + c];
    const double hn = sqrt(nn);
    double2 *col = s.H + (GM_M + 1) * j;
    // previous rotations
    for (int i = 0; i < j; i++) {
        const double c = s.cs[i];
        const double2 sn = s.sn[i];
        const double2 a = col[i], b = col[i + 1];
        const double2 sb = cmul(sn, b);
        const double2 sa = cmulc(sn, a);   // conj(s) a
        col[i] = make_double2(c * a.x + sb.x, c * a.y + sb.y);
        col[i + 1] = make_double2(c * b.x - sa.x, c * b.y - sa.y);
    }
    // new rotation zeroing h_{j+1,j} = hn (real, >= 0)
    const double2 a = col[j];
    const double aa = hypot(a.x, a.y);
    const double r = hypot(aa, hn);
    double c;
    double2 sn;
    double2 rr;
    if (aa == 0.0) {
        c = 0.0;
        sn = make_double2(1.0, 0.0);
        rr = make_double2(hn, 0.0);
    } else {
        c = aa / r;
        const double2 ph = make_double2(a.x / aa, a.y / aa);
        sn = make_double2(ph.x * hn / r, ph.y * hn / r);
        rr = make_double2(ph.x * r, ph.y * r);
    }
    s.cs[j] = c;
    s.sn[j] = sn;
    col[j] = rr;
    col[j + 1] = make_double2(0.0, 0.0);
    const double2 gj = s.g[j];
    const double2 sg = cmulc(sn, gj);
    s.g[j + 1] = make_double2(-sg.x, -sg.y);
    s.g[j] = make_double2(c * gj.x, c * gj.y);
    s.res = hypot(s.g[j + 1].x, s.g[j + 1].y);
    s.j = j + 1;
    const bool breakdown = !(hn > 1e-300 * (s.beta > 0 ? s.beta : 1.0));
    s.inv_h = breakdown ? 0.0 : 1.0 / hn;
    if (s.res <= s.tolabs || j + 1 == GM_M || breakdown || !(r > 0.0)) {
        s.stop = 1;
        *ctl_skip(ctl, f) = 1;   // the triangular solves skip this frequency too
    }
}

// v_{j+1} = w / h_{j+1,j} and its complex64 copy for the next preconditioner solve.
__global__ void __launch_bounds__(256) k_gm_normalize(int N, int B, int j, double2 *__restrict__ V,
                                                      const double2 *__restrict__ wb, float2 *__restrict__ rfb,
                                                      int vstride, const GmState *__restrict__ st) {
    const int f = blockIdx.y;
    if (st[f].stop) return;
    const int n = blockIdx.x * 256 + threadIdx.x;
    if (n >= N) return;
    const double inv = st[f].inv_h;
    const double2 w = wb[(size_t)N * f + n];
    const double2 v = make_double2(w.x * inv, w.y * inv);
    V[((size_t)(j + 1) * B + f) * N + n] = v;
    rfb[(size_t)vstride * f + n] = make_float2((float)v.x, (float)v.y);
}

// y = R^-1 g (R = rotated H, k = s.j steps), one thread per frequency.
__global__ void k_gm_solve_y(int B, GmState *__restrict__ st, const char *__restrict__ ctl,
                             const int *__restrict__ active) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= B) return;
    GmState &s = st[f];
    if (*reinterpret_cast<const int *>(ctl + 64 * f + 28) || !active[f]) {   // converged before the cycle, or empty
        s.j = 0;
        return;
    }
    const int k = s.j;
    for (int i = k - 1; i >= 0; i--) {
        double2 t = s.g[i];
        for (int q = i + 1; q < k; q++) {
            const double2 hy = cmul(s.H[i + (GM_M + 1) * q], s.y[q]);
            t.x -= hy.x;
            t.y -= hy.y;
        }
        const double2 d = s.H[i + (GM_M + 1) * i];
        const double den = d.x * d.x + d.y * d.y;
        s.y[i] = den > 0.0 ? make_double2((t.x * d.x + t.y * d.y) / den, (t.y * d.x - t.x * d.y) / den)
                           : make_double2(0.0, 0.0);
    }
}

// x += Zm y over the k = s.j stored preconditioned vectors.
__global__ void __launch_bounds__(256) k_gm_update_x(int N, int B, const double2 *__restrict__ Zm,
                                                     double2 *__restrict__ xb, const GmState *__restrict__ st) {
    const int f = blockIdx.y;
    const int k = st[f].j;
    if (k == 0) return;
    const int n = blockIdx.x * 256 + threadIdx.x;
    if (n >= N) return;
    double2 acc = xb[(size_t)N * f + n];
    for (int i = 0; i < k; i++) {
        const double2 t = cmul(Zm[((size_t)i * B + f) * N + n], st[f].y[i]);
        acc.x += t.x;
        acc.y += t.y;
    }
    xb[(size_t)N * f + n] = acc;
}

// Before the true residual: frequencies not yet converged take part again.
__global__ void k_gm_reset_skip(int B, char *__restrict__ ctl, const int *__restrict__ active) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= B) return;
    *ctl_skip(ctl, f) = *ctl_conv(ctl, f) || !active[f];
}

// ---------------------------------------------------------------------------
// y_f = Z_f x_f for a symmetric Z_f (full column-major storage, upper
// triangle read once).  Tile t = (I, J), I <= J, of ST x ST entries
// (t = J (J + 1) / 2 + I): rows I, columns J.  It contributes Z_IJ x_J to y_I
// and, off the diagonal, Z_IJ^T x_I to y_J; both partial vectors go to
// P[f][t][2][ST] and k_symv_reduce adds them in a fixed order, so the
// product is bit-reproducible.
//
// k_symv_ring: one persistent CTA per SM walks its (tile, frequency) items;
// every tile arrives as four chunks of 32 columns x 128 rows (64 KB, one TMA
// box of the map of Z; zeros past row and column N) through a ring of three
// stages that thread 0 refills in the CTA's item order, so the next chunks
// -- also those of the next items -- are in flight while the CTA works.  Warp
// w takes columns 4 w .. 4 w + 3 of each chunk (lane l its rows l + 32 q)
// and reduces their four column sums across the warp together (each halving
// step exchanges half of the values still held).  A frequency whose flag
// (flags[f * fstride]) is set is skipped.
// ---------------------------------------------------------------------------
constexpr int ST = 128;

__device__ __forceinline__ void tile_of(int t, int &I, int &J) {
    int j = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((j + 1) * (j + 2) / 2 <= t) j++;
    while (j * (j + 1) / 2 > t) j--;
    J = j;
    I = t - j * (j + 1) / 2;
}

__device__ __forceinline__ double2 shfl_xor2(double2 v, int o) {
    return make_double2(__shfl_xor_sync(0xffffffffu, v.x, o), __shfl_xor_sync(0xffffffffu, v.y, o));
}

__device__ __forceinline__ void cadd(double2 &a, const double2 &b) {
    a.x += b.x;
    a.y += b.y;
}

constexpr int SC = 32;                                  // columns per chunk
constexpr int SRING = 3;                                // stages of the chunk ring
constexpr uint32_t SCHUNK = ST * SC * sizeof(double2);  // 64 KB
constexpr size_t SYMV_SMEM = SRING * SCHUNK + 1024 + 64;

__global__ void __launch_bounds__(256, 1) k_symv_ring(const __grid_constant__ CUtensorMap zmap, int N, int ntiles,
                                                      int B, const double2 *__restrict__ xb, double2 *__restrict__ P,
                                                      const int *__restrict__ flags, int fstride, char *ctl) {
    using namespace efie_tma;
    extern __shared__ unsigned char dsm[];
    __shared__ double2 rsum[8][ST];
    __shared__ double2 csum[ST];
    __shared__ int fail;
    unsigned char *ring = dsm + (((smem_u32(dsm) + 1023u) & ~1023u) - smem_u32(dsm));
    uint64_t *full = reinterpret_cast<uint64_t *>(ring + SRING * SCHUNK);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int G = gridDim.x, items = ntiles * B;
    auto live = [&](int it) -> bool { return !flags[(size_t)(it / ntiles) * fstride]; };
    // producer state (thread 0): chunk p_c of item p_it is the next to load
    int p_it = blockIdx.x, p_c = 0, issued = 0;
    auto produce = [&]() {
        if (p_it >= items) return;
        const int f = p_it / ntiles, t = p_it - f * ntiles;
        int I, J;
        tile_of(t, I, J);
        uint64_t *bar = full + issued % SRING;
        mbar_expect_tx(bar, SCHUNK);
        tma_load_3d(&zmap, ring + (issued % SRING) * SCHUNK, 2 * I * ST, J * ST + p_c * SC, f, bar);
        issued++;
        if (++p_c == ST / SC) {
            p_c = 0;
            for (p_it += G; p_it < items && !live(p_it); p_it += G) {
            }
        }
    };
    if (tid == 0) {
        for (int s = 0; s < SRING; s++) mbar_init(full + s, 1);
        mbar_init_fence();
        fail = 0;
        while (p_it < items && !live(p_it)) p_it += G;
        for (int s = 0; s < SRING; s++) produce();
    }
    __syncthreads();
    int cc = 0;
    for (int it = blockIdx.x; it < items; it += G) {
        if (!live(it)) continue;
        const int f = it / ntiles, t = it - f * ntiles;
        int I, J;
        tile_of(t, I, J);
        const double2 *x = xb + (size_t)N * f;
        const int r0 = I * ST, c0 = J * ST;
        const bool offdiag = I != J;
        double2 xr[4], rs[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int m = r0 + lane + 32 * q;
            xr[q] = m < N ? x[m] : make_double2(0.0, 0.0);
            rs[q] = make_double2(0.0, 0.0);
        }
#pragma unroll 1
        for (int c = 0; c < ST / SC; c++) {
            if (!mbar_wait_bounded(full + cc % SRING, (uint32_t)(cc / SRING) & 1u)) fail = 1;
            const double2 *chunk = reinterpret_cast<const double2 *>(ring + (cc % SRING) * SCHUNK);
            const int cb = c * SC + warp * 4;   // first column of the warp's group within the tile
            if (!fail) {
                double2 a[4][4], xn[4];
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int n = c0 + cb + j;
                    xn[j] = n < N ? x[n] : make_double2(0.0, 0.0);
#pragma unroll
                    for (int q = 0; q < 4; q++) a[j][q] = chunk[(warp * 4 + j) * ST + lane + 32 * q];
                }
                double2 cs[4];
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    cs[j] = make_double2(0.0, 0.0);
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const double2 v = a[j][q];
                        rs[q].x += v.x * xn[j].x - v.y * xn[j].y;
                        rs[q].y += v.x * xn[j].y + v.y * xn[j].x;
                        cs[j].x += v.x * xr[q].x - v.y * xr[q].y;
                        cs[j].y += v.x * xr[q].y + v.y * xr[q].x;
                    }
                }
                if (offdiag) {   // block-uniform
                    // lanes with bit 4 set keep columns 2, 3 (send 0, 1), the others keep 0, 1
                    const bool b4 = lane & 16, b3 = lane & 8;
                    double2 k0 = b4 ? cs[2] : cs[0], k1 = b4 ? cs[3] : cs[1];
                    cadd(k0, shfl_xor2(b4 ? cs[0] : cs[2], 16));
                    cadd(k1, shfl_xor2(b4 ? cs[1] : cs[3], 16));
                    // bit 3 picks one of the two
                    double2 k = b3 ? k1 : k0;
                    cadd(k, shfl_xor2(b3 ? k0 : k1, 8));
                    cadd(k, shfl_xor2(k, 4));
                    cadd(k, shfl_xor2(k, 2));
                    cadd(k, shfl_xor2(k, 1));
                    // lane 8 c holds column cb + c (c = 2 b4 + b3)
                    if ((lane & 7) == 0) csum[cb + (lane >> 3)] = k;
                }
            }
            __syncthreads();   // every warp is done with the stage
            if (fail) {
                // a chunk never arrived: every frequency of the launch falls back
                if (tid < B) atomicExch(reinterpret_cast<int *>(ctl + 64 * tid + 36), 3);
                if (tid == 0)
                    for (int k = cc + 1; k < issued; k++)
                        if (!mbar_wait_bounded(full + k % SRING, (uint32_t)(k / SRING) & 1u)) break;
                return;
            }
            if (tid == 0) produce();
            cc++;
        }
#pragma unroll
        for (int q = 0; q < 4; q++) rsum[warp][lane + 32 * q] = rs[q];
        __syncthreads();
        double2 *out = P + ((size_t)f * ntiles + t) * 2 * ST;
        if (tid < ST) {
            double2 v = make_double2(0.0, 0.0);
            for (int w = 0; w < 8; w++) {
                v.x += rsum[w][tid].x;
                v.y += rsum[w][tid].y;
            }
            out[tid] = v;
        } else if (offdiag) {
            out[tid] = csum[tid - ST];
        }
        __syncthreads();   // rsum and csum are free for the next item
    }
}

// y_I = sum_{J >= I} (row part of tile (I, J)) + sum_{J < I} (column part of tile (J, I))
__global__ void __launch_bounds__(ST) k_symv_reduce(int N, int nb, const double2 *__restrict__ P,
                                                    double2 *__restrict__ yb, const int *__restrict__ flags,
                                                    int fstride) {
    const int f = blockIdx.y;
    if (flags[(size_t)f * fstride]) return;
    const int I = blockIdx.x, r = threadIdx.x, m = I * ST + r;
    const size_t ntiles = (size_t)nb * (nb + 1) / 2;
    const double2 *Pf = P + (size_t)f * ntiles * 2 * ST;
    double2 acc = make_double2(0.0, 0.0);
    for (int J = 0; J < nb; J++) {
        double2 v;
        if (J < I) v = Pf[((size_t)I * (I + 1) / 2 + J) * 2 * ST + ST + r];   // tile (J, I), column part
        else v = Pf[((size_t)J * (J + 1) / 2 + I) * 2 * ST + r];             // tile (I, J), row part
        acc.x += v.x;
        acc.y += v.y;
    }
    if (m < N) yb[(size_t)N * f + m] = acc;
}

inline unsigned cdiv(size_t a, size_t b) { return (unsigned)((a + b - 1) / b); }

// the stop flags of the batch in one array (one read-back per poll)
__global__ void k_gm_stop_flags(int B, const GmState *__restrict__ st, int *__restrict__ out) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f < B) out[f] = st[f].stop;
}

// the map of Z (all slots) for k_symv_ring: doubles [B][N][2N] (innermost
// first: re/im of a row, column, slot), boxes of 128 rows x 32 columns
efie_status symv_map(SolveWork &w, const void *Z, size_t zstride) {
    if (w.zmap_base == Z && w.zmap_stride == zstride && w.zmap_n == w.N && w.zmap_b == w.B) return EFIE_OK;
    const cuuint64_t dims[3] = {2 * (cuuint64_t)w.N, (cuuint64_t)w.N, (cuuint64_t)w.B};
    const cuuint64_t strides[2] = {sizeof(double2) * (cuuint64_t)w.N, sizeof(double2) * (cuuint64_t)zstride};
    const cuuint32_t box[3] = {2 * ST, SC, 1};
    EFIE_TRY(efie_encode_tiled(w.zmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<void *>(Z), dims, strides, box,
                               CU_TENSOR_MAP_SWIZZLE_NONE));
    w.zmap_base = Z;
    w.zmap_stride = zstride;
    w.zmap_n = w.N;
    w.zmap_b = w.B;
    return EFIE_OK;
}

efie_status symv(efie_ctx *ctx, SolveWork &w, const void *Z, size_t zstride, const double2 *x, double2 *y,
                 const int *flags, int fstride) {
    const int nb = (w.N + ST - 1) / ST;
    const size_t ntiles = (size_t)nb * (nb + 1) / 2;
    EFIE_TRY(w.spart.reserve(sizeof(double2) * ntiles * 2 * ST * w.B));
    EFIE_TRY(symv_map(w, Z, zstride));
    EFIE_CUDA(cudaFuncSetAttribute(k_symv_ring, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SYMV_SMEM));
    cudaStream_t s = ctx->stream;
    const int grid = (int)std::min<size_t>((size_t)ctx->num_sms, ntiles * w.B);
    k_symv_ring<<<grid, 256, SYMV_SMEM, s>>>(*reinterpret_cast<const CUtensorMap *>(w.zmap), w.N, (int)ntiles, w.B,
                                             x, w.spart.as<double2>(), flags, fstride, w.ctl.as<char>());
    k_symv_reduce<<<dim3(nb, w.B), ST, 0, s>>>(w.N, nb, w.spart.as<double2>(), y, flags, fstride);
    EFIE_CUDA(cudaGetLastError());
    return EFIE_OK;
}

efie_status gm_workspace(SolveWork &w) {
    const size_t NB = (size_t)w.N * w.B;
    w.gnch = (int)cdiv(w.N, ROWS);
    EFIE_TRY(w.gV.reserve(sizeof(double2) * NB * (GM_M + 1)));
    EFIE_TRY(w.gZ.reserve(sizeof(double2) * NB * GM_M));
    EFIE_TRY(w.gw.reserve(sizeof(double2) * NB));
    EFIE_TRY(w.gpart.reserve(sizeof(double2) * (size_t)w.B * w.gnch * (GM_M + 1) + sizeof(double) * w.B * w.gnch));
    EFIE_TRY(w.gst.reserve(sizeof(GmState) * w.B));
    EFIE_TRY(w.gflags.reserve(sizeof(int) * w.B));
    if (w.zsym) {
        const int nb = (w.N + ST - 1) / ST;
        EFIE_TRY(w.spart.reserve(sizeof(double2) * ((size_t)nb * (nb + 1) / 2) * 2 * ST * w.B));
    }
    return EFIE_OK;
}

}  // namespace

efie_status efie_mixed_gmres(efie_ctx *ctx, SolveWork &w, const void *Z, size_t zstride, const void *b, void *x,
                             double bnorm, double tol, int max_iter, const int *active_host, RefineResult *res,
                             bool x0_given) {
    cudaStream_t s = ctx->stream;
    KernelLog &log = ctx->log;
    const int N = w.N, B = w.B;
    EFIE_TRY(gm_workspace(w));
    const int nch = w.gnch;
    char *ctl = w.ctl.as<char>();
    float2 *rf = w.vec.as<float2>(), *yv = rf + (size_t)w.vstride * B, *dv = yv + (size_t)w.vstride * B;
    double2 *V = w.gV.as<double2>(), *Zm = w.gZ.as<double2>(), *wv = w.gw.as<double2>();
    double2 *part = w.gpart.as<double2>();
    double *npart = reinterpret_cast<double *>(part + (size_t)B * nch * (GM_M + 1));
    GmState *st = w.gst.as<GmState>();
    const int *active = w.active.as<int>();
    int nact = 0;
    for (int f = 0; f < B; f++) nact += active_host[f] ? 1 : 0;
    const double zbytes = 16.0 * (double)N * N, lubytes = 8.0 * (double)N * N;
    const double tol_inner = 0.5 * tol;
    const int *ctl_skip0 = reinterpret_cast<const int *>(ctl + 32);   // ctl skip flag of slot f: [16 f]
    auto residual = [&]() -> efie_status {
        if (!w.zsym) return efie_true_residual(ctx, w, Z, zstride, x, b, tol, V, nact);
        size_t tk = log.begin(s);
        EFIE_TRY(symv(ctx, w, Z, zstride, static_cast<const double2 *>(x), wv, ctl_skip0, 16));
        log.end(EFIE_K_RESIDUAL, s, tk, 8.0 * (double)N * N * nact, 2);
        return efie_residual_finish(ctx, w, wv, b, tol, V, nact);
    };
    EFIE_TRY(efie_refine_init(ctx, w, x, bnorm, !x0_given));
    // r0 = b - Z x0, stored at V slot 0 too; for x0 = 0 without the product
    if (x0_given || !w.zsym) {
        EFIE_TRY(residual());
    } else {
        EFIE_CUDA(cudaMemsetAsync(wv, 0, sizeof(double2) * (size_t)N * B, s));
        EFIE_TRY(efie_residual_finish(ctx, w, wv, b, tol, V, nact));
    }
    std::vector<char> hctl(64 * (size_t)B);
    std::vector<int> hstop(B);
    int matvecs = 0;
    // frequencies still iterating as of the last stop-flag poll: the work the
    // in-cycle launches count (a stopped frequency's CTAs return at once)
    int nrun = nact;
    bool all_conv = false, failed = false;
    const dim3 vg(cdiv(N, 256), B), og(nch, B), mg(cdiv(N, 32), B);
    while (!all_conv && !failed && matvecs < max_iter) {
        size_t tok = log.begin(s);
        k_gm_start<<<vg, 256, 0, s>>>(N, B, V, rf, w.vstride, st, ctl, tol_inner, active);
        EFIE_CUDA(cudaGetLastError());
        log.end(EFIE_K_OTHER, s, tok, 0.0);
        int j = 0;
        for (; j < GM_M && matvecs < max_iter; j++) {
            const int epoch = ++w.epoch;
            double2 *zj = Zm + (size_t)j * B * N;
            EFIE_CUDA(cudaMemsetAsync(zj, 0, sizeof(double2) * (size_t)B * N, s));
            tok = log.begin(s);
            EFIE_TRY(efie_trsv(ctx, w, true, rf, yv, nullptr, epoch));
            EFIE_TRY(efie_trsv(ctx, w, false, yv, dv, zj, epoch));
            log.end(EFIE_K_TRSV, s, tok, lubytes * nrun, 2);
            tok = log.begin(s);
            if (w.zsym) {
                EFIE_TRY(symv(ctx, w, Z, zstride, zj, wv, &st[0].stop, (int)(sizeof(GmState) / sizeof(int))));
                log.end(EFIE_K_RESIDUAL, s, tok, 0.5 * zbytes * nrun, 2);
            } else {
                k_gm_matvec<<<mg, 256, 0, s>>>(N, static_cast<const double2 *>(Z), zstride, zj, wv, st);
                EFIE_CUDA(cudaGetLastError());
                log.end(EFIE_K_RESIDUAL, s, tok, zbytes * nrun);
            }
            tok = log.begin(s);
            k_gm_zero_col<<<B, GM_M + 1, 0, s>>>(B, j, st);
            for (int pass = 0; pass < 2; pass++) {
                k_gm_dot<<<og, ROWS, 0, s>>>(N, B, j + 1, V, wv, part, st);
                k_gm_axpy<<<og, ROWS, 0, s>>>(N, B, j + 1, j, V, wv, part, st, pass == 1 ? npart : nullptr);
            }
            k_gm_arnoldi<<<cdiv(B, 32), 32, 0, s>>>(B, j, nch, npart, st, ctl);
            k_gm_normalize<<<vg, 256, 0, s>>>(N, B, j, V, wv, rf, w.vstride, st);
            EFIE_CUDA(cudaGetLastError());
            log.end(EFIE_K_OTHER, s, tok, 32.0 * (double)N * (j + 1) * 2 * nrun, 7);
            matvecs++;
            if (j >= 2) {
                // a poll costs one synchronisation (tens of us) against a step
                // of the whole batch (milliseconds at large N)
                bool all_stop = true;
                tok = log.begin(s);
                k_gm_stop_flags<<<cdiv(B, 32), 32, 0, s>>>(B, st, w.gflags.as<int>());
                EFIE_CUDA(cudaGetLastError());
                log.end(EFIE_K_OTHER, s, tok, 0.0);
                EFIE_CUDA(cudaMemcpyAsync(hstop.data(), w.gflags.p, sizeof(int) * B, cudaMemcpyDeviceToHost, s));
                EFIE_CUDA(cudaStreamSynchronize(s));
                nrun = 0;
                for (int f = 0; f < B; f++)
                    if (active_host[f] && !hstop[f]) all_stop = false, nrun++;
                if (all_stop) {
                    j++;
                    break;
                }
            }
        }
        tok = log.begin(s);
        k_gm_solve_y<<<cdiv(B, 32), 32, 0, s>>>(B, st, ctl, active);
        k_gm_update_x<<<vg, 256, 0, s>>>(N, B, Zm, static_cast<double2 *>(x), st);
        k_gm_reset_skip<<<cdiv(B, 32), 32, 0, s>>>(B, ctl, active);
        EFIE_CUDA(cudaGetLastError());
        log.end(EFIE_K_OTHER, s, tok, 0.0, 3);
        // true residual; a restart begins from it
        EFIE_TRY(residual());
        EFIE_CUDA(cudaMemcpyAsync(hctl.data(), ctl, 64 * (size_t)B, cudaMemcpyDeviceToHost, s));
        EFIE_CUDA(cudaStreamSynchronize(s));
        all_conv = true;
        nrun = 0;
        for (int f = 0; f < B; f++) {
            if (!active_host[f]) continue;
            const char *c = hctl.data() + 64 * f;
            if (*reinterpret_cast<const int *>(c + 36)) failed = true;
            if (!*reinterpret_cast<const int *>(c + 28)) all_conv = false, nrun++;
        }
    }
    res->iters = matvecs;
    for (int f = 0; f < B; f++) {
        const char *c = hctl.data() + 64 * f;
        res->relres[f] = reinterpret_cast<const double *>(c)[2];
        res->converged[f] = *reinterpret_cast<const int *>(c + 28) != 0;
        res->err[f] = *reinterpret_cast<const int *>(c + 36);
    }
    return EFIE_OK;
}
