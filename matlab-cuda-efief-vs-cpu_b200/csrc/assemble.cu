// FP64 impedance-matrix assembly on sm_100a.
//
// The reference evaluates every RWG pair (m,n) by looping over its four
// triangle pairs and recomputing the quadrature (kernel_Z_fastquad,
// patch_sweep_fastquad_cuda.cu:347-412).  A triangle pair is shared by up to
// 3x3 RWG pairs, so here the quadrature runs once per triangle pair and
// produces eight complex moments in local coordinates (rho = r - o_t):
//   S0 = sum W G,  S1 = sum W G rho_i,  S2 = sum W G rho'_j,  S3 = sum W G rho_i.rho'_j
// With the RWG basis written as f = c (r - v), div = 2c
// (rwg_eval_on_triangle.m:10-28: plus side c = s+ l/(2A+), v = r+; minus side
// c = -s- l/(2A-), v = r-), every RWG pair entry is
//   Ivec = c_m c_n [S3 - d_n.S1 - d_m.S2 + (d_m.d_n) S0],  Isca = 4 c_m c_n S0
// with d = v - o.  Pair regimes follow Z_entry (CPU_FAST.m:48-54): self when
// t1 == t2, near when nearMat(t1,t2), else regular.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "efie_internal.h"

namespace {

constexpr double kPi = 3.141592653589793238462643383279502884;

struct Mom {
    double v[16];  // S0(re,im) S1x S1y S1z S2x S2y S2z S3 (re,im each)
};

__device__ __forceinline__ void green(double kr, double ki, double R, double &gr, double &gi) {
    // exp(-j k R)/(4 pi R), k = kr + j ki  (patch_sweep_fastquad_cuda.cu:60-71)
    double s, c;
    sincos(kr * R, &s, &c);
    double inv = 1.0 / (4.0 * kPi * R);
    if (ki != 0.0) inv *= exp(ki * R);
    gr = c * inv;
    gi = -s * inv;
}

__device__ __forceinline__ size_t pair_slot(int t1, int t2, int Nt, bool sym) {
    if (!sym) return (size_t)t1 + (size_t)Nt * (size_t)t2;
    int lo = min(t1, t2), hi = max(t1, t2);
    return (size_t)hi * (size_t)(hi + 1) / 2 + (size_t)lo;
}

// Triangle-pair moments of the pair (t1, t2), t1 the triangle of rho and t2
// that of rho': S0 = int G, S1 = int G rho, S2 = int G rho', S3 = int G
// rho.rho' (complex; rho, rho' relative to each triangle's origin), stored
// component-major at p[c * stride + q] for pair slot q, so consecutive
// threads (consecutive slots) store and load coalesced runs of 16 bytes.
//
// Edge-combination form (tri_d set): an RWG side on triangle t contributes
// c (rho - d) with d one of at most three free-vertex vectors of t (its slot
// l), so the pair's whole contribution to an entry is c_m c_n Q[l1][l2] with
//     Q[l1][l2] = alpha (S3 - d2.S1 - d1.S2 + (d1.d2) S0) + beta 4 S0,
// nine complex values per pair, p[(3 l1 + l2) * stride + q]: the gather then
// reads one value per triangle pair instead of eight.  Otherwise the eight
// moments themselves (c = S0, S1x, S1y, S1z, S2x, S2y, S2z, S3).
struct MomStore {
    double2 *p;
    size_t stride;
    const double4 *tri_d;   // [Nt][3] free-vertex vectors per slot, or null
    double alr, ali, ber, bei;
};

__device__ __forceinline__ void store_mom(const MomStore &M, size_t slot, int t1, int t2, const double *a) {
    if (!M.tri_d) {
#pragma unroll
        for (int i = 0; i < 8; i++) M.p[(size_t)i * M.stride + slot] = make_double2(a[2 * i], a[2 * i + 1]);
        return;
    }
    const double s0r = 4.0 * a[0], s0i = 4.0 * a[1];
    const double bsr = M.ber * s0r - M.bei * s0i, bsi = M.ber * s0i + M.bei * s0r;   // beta 4 S0
#pragma unroll
    for (int l1 = 0; l1 < 3; l1++) {
        const double4 d1 = M.tri_d[3 * (size_t)t1 + l1];
        // S3 - d1.S2 and S1 - d1 S0
        const double ar = a[14] - (d1.x * a[8] + d1.y * a[10] + d1.z * a[12]);
        const double ai = a[15] - (d1.x * a[9] + d1.y * a[11] + d1.z * a[13]);
        const double bxr = a[2] - d1.x * a[0], bxi = a[3] - d1.x * a[1];
        const double byr = a[4] - d1.y * a[0], byi = a[5] - d1.y * a[1];
        const double bzr = a[6] - d1.z * a[0], bzi = a[7] - d1.z * a[1];
#pragma unroll
        for (int l2 = 0; l2 < 3; l2++) {
            const double4 d2 = M.tri_d[3 * (size_t)t2 + l2];
            const double ivr = ar - (d2.x * bxr + d2.y * byr + d2.z * bzr);
            const double ivi = ai - (d2.x * bxi + d2.y * byi + d2.z * bzi);
            M.p[(size_t)(3 * l1 + l2) * M.stride + slot] =
                make_double2((M.alr * ivr - M.ali * ivi) + bsr, (M.alr * ivi + M.ali * ivr) + bsi);
        }
    }
}

// ---------------------------------------------------------------------------
// Regular pairs: one thread per triangle pair, NQ points per triangle.
// Block = 32 (t1) x 8 (t2).  Regular quadrature of CPU_FAST.m:63-89 with
// R = max(R, 1e-15).
// ---------------------------------------------------------------------------
template <int NQ>
__global__ void __launch_bounds__(256) k_regular_moments(
    int Nt, bool sym, const double4 *__restrict__ origin, const double4 *__restrict__ pts,
    const uint8_t *__restrict__ skip, double kr, double ki, MomStore mom) {
    __shared__ double4 sp[8][NQ];
    __shared__ double4 so[8];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int t1 = blockIdx.x * 32 + tx;
    const int t2b = blockIdx.y * 8;
    if (sym && blockIdx.x * 32 > t2b + 7) return;  // whole tile below the diagonal
    for (int i = threadIdx.x; i < 8 * NQ; i += blockDim.x) {
        int tt = t2b + i / NQ;
        sp[i / NQ][i % NQ] = tt < Nt ? pts[(size_t)tt * NQ + i % NQ] : make_double4(0, 0, 0, 0);
    }
    if (threadIdx.x < 8) {
        int tt = t2b + threadIdx.x;
        so[threadIdx.x] = tt < Nt ? origin[tt] : make_double4(0, 0, 0, 0);
    }
    __syncthreads();
    const int t2 = t2b + ty;
    if (t1 >= Nt || t2 >= Nt) return;
    if (sym && t1 > t2) return;
    if (skip[(size_t)t1 + (size_t)Nt * t2]) return;
    double4 p1[NQ];
#pragma unroll
    for (int p = 0; p < NQ; p++) p1[p] = pts[(size_t)t1 * NQ + p];
    const double4 o1 = origin[t1], o2 = so[ty];
    const double dox = o1.x - o2.x, doy = o1.y - o2.y, doz = o1.z - o2.z;
    double m[16];
#pragma unroll
    for (int i = 0; i < 16; i++) m[i] = 0.0;
#pragma unroll 1
    for (int q = 0; q < NQ; q++) {
        const double4 pq = sp[ty][q];
        const double ax = dox - pq.x, ay = doy - pq.y, az = doz - pq.z;
        double t0r = 0, t0i = 0, t1r[3] = {0, 0, 0}, t1i[3] = {0, 0, 0};
#pragma unroll
        for (int p = 0; p < NQ; p++) {
            const double dx = ax + p1[p].x, dy = ay + p1[p].y, dz = az + p1[p].z;
            double R = sqrt(dx * dx + dy * dy + dz * dz);
            R = fmax(R, 1e-15);
            double gr, gi;
            green(kr, ki, R, gr, gi);
            gr *= p1[p].w;
            gi *= p1[p].w;
            t0r += gr;
            t0i += gi;
            t1r[0] += gr * p1[p].x; t1i[0] += gi * p1[p].x;
            t1r[1] += gr * p1[p].y; t1i[1] += gi * p1[p].y;
            t1r[2] += gr * p1[p].z; t1i[2] += gi * p1[p].z;
        }
        const double w = pq.w;
        m[0] += w * t0r; m[1] += w * t0i;
        m[2] += w * t1r[0]; m[3] += w * t1i[0];
        m[4] += w * t1r[1]; m[5] += w * t1i[1];
        m[6] += w * t1r[2]; m[7] += w * t1i[2];
        m[8] += w * t0r * pq.x; m[9] += w * t0i * pq.x;
        m[10] += w * t0r * pq.y; m[11] += w * t0i * pq.y;
        m[12] += w * t0r * pq.z; m[13] += w * t0i * pq.z;
        m[14] += w * (pq.x * t1r[0] + pq.y * t1r[1] + pq.z * t1r[2]);
        m[15] += w * (pq.x * t1i[0] + pq.y * t1i[1] + pq.z * t1i[2]);
    }
    store_mom(mom, pair_slot(t1, t2, Nt, sym), t1, t2, m);
}

// Several frequencies at once (F = 2..4, equally spaced: k_f = k0 + f dk).
// Per point pair R, 1/(4 pi R) and the weights are shared, e^{-j k0 R} and
// e^{-j dk R} take one sincos each (and exp for lossy media), and every
// further frequency costs one complex multiplication: e^{-j k_f R} =
// e^{-j k0 R} (e^{-j dk R})^f.  The pair values go to each frequency's store.
//
// Cost per point pair, shared by the F frequencies: R and 1/R come from one
// reciprocal square root of R^2 (R = R^2 rsqrt(R^2)) instead of a square
// root and a division; the phase step dk R of a dense sweep is small, and for
// |dk R| <= 1/2 its cosine and sine are the Maclaurin series through x^14 and
// x^15 (truncation below 1e-18, Horner in x^2), larger steps take sincos.
// With symmetric pairs the launch covers the tiles on or above the diagonal
// only (a host-built list of (t1 block, t2 block)); the free-vertex vectors
// of the tile's 40 triangles are staged in shared memory with the points, so
// the nine edge combinations per frequency read them there.
struct MomStores {
    MomStore s[4];
};

// cos x and sin x for |x| <= 1/2 from their Maclaurin series:
// cos x = sum (-1)^n x^{2n} / (2n)!, sin x = x sum (-1)^n x^{2n} / (2n+1)!
__device__ __forceinline__ void small_sincos(double x, double &sn, double &cs) {
    const double u = x * x;
    double c = 1.0 / 87178291200.0;                        // 1/14!
    c = fma(c, -u, 1.0 / 479001600.0);                      // 1/12!
    c = fma(c, -u, 1.0 / 3628800.0);                        // 1/10!
    c = fma(c, -u, 1.0 / 40320.0);                          // 1/8!
    c = fma(c, -u, 1.0 / 720.0);                            // 1/6!
    c = fma(c, -u, 1.0 / 24.0);                             // 1/4!
    c = fma(c, -u, 0.5);                                    // 1/2!
    cs = fma(c, -u, 1.0);
    double t = 1.0 / 1307674368000.0;                       // 1/15!
    t = fma(t, -u, 1.0 / 6227020800.0);                     // 1/13!
    t = fma(t, -u, 1.0 / 39916800.0);                       // 1/11!
    t = fma(t, -u, 1.0 / 362880.0);                         // 1/9!
    t = fma(t, -u, 1.0 / 5040.0);                           // 1/7!
    t = fma(t, -u, 1.0 / 120.0);                            // 1/5!
    t = fma(t, -u, 1.0 / 6.0);                              // 1/3!
    sn = fma(x * u, -t, x);
}

// the nine edge combinations of one pair and frequency from its moments,
// with the free-vertex vectors d1[3] (triangle t1) and d2[3] (t2) at hand
__device__ __forceinline__ void store_combo(const MomStore &M, size_t slot, const double4 *d1s, const double4 *d2s,
                                            const double *a) {
    const double s0r = 4.0 * a[0], s0i = 4.0 * a[1];
    const double bsr = M.ber * s0r - M.bei * s0i, bsi = M.ber * s0i + M.bei * s0r;   // beta 4 S0
#pragma unroll
    for (int l1 = 0; l1 < 3; l1++) {
        const double4 d1 = d1s[l1];
        const double ar = a[14] - (d1.x * a[8] + d1.y * a[10] + d1.z * a[12]);
        const double ai = a[15] - (d1.x * a[9] + d1.y * a[11] + d1.z * a[13]);
        const double bxr = a[2] - d1.x * a[0], bxi = a[3] - d1.x * a[1];
        const double byr = a[4] - d1.y * a[0], byi = a[5] - d1.y * a[1];
        const double bzr = a[6] - d1.z * a[0], bzi = a[7] - d1.z * a[1];
#pragma unroll
        for (int l2 = 0; l2 < 3; l2++) {
            const double4 d2 = d2s[l2];
            const double ivr = ar - (d2.x * bxr + d2.y * byr + d2.z * bzr);
            const double ivi = ai - (d2.x * bxi + d2.y * byi + d2.z * bzi);
            __stcs(M.p + (size_t)(3 * l1 + l2) * M.stride + slot,
                   make_double2((M.alr * ivr - M.ali * ivi) + bsr, (M.alr * ivi + M.ali * ivr) + bsi));
        }
    }
}

// t2 rows per CTA of the multi-frequency kernel: 32 x 4 pairs in 128 threads,
// so that two CTAs share an SM (the 64 accumulators of four frequencies allow
// eight warps) and one's loads and stores overlap the other's arithmetic
// (32 x 2 tiles in 64 threads measured the same)
constexpr int MF_RY = 4;

template <int NQ, int F>
__global__ void __launch_bounds__(32 * MF_RY) k_regular_moments_mf(
    int Nt, bool sym, const int2 *__restrict__ tiles, const double4 *__restrict__ origin,
    const double4 *__restrict__ pts, const uint8_t *__restrict__ skip, double kr0, double ki0, double dkr,
    double dki, MomStores ms) {
    __shared__ double4 sp[MF_RY][NQ];
    __shared__ double4 so[MF_RY];
    __shared__ double4 sd1[32][3], sd2[MF_RY][3];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    int bx = blockIdx.x, by = blockIdx.y;
    if (tiles) {
        const int2 tl = tiles[blockIdx.x];
        bx = tl.x;
        by = tl.y;
    }
    const int t1 = bx * 32 + tx;
    const int t2b = by * MF_RY;
    if (sym && bx * 32 > t2b + MF_RY - 1) return;  // whole tile below the diagonal
    const double4 *tri_d = ms.s[0].tri_d;
    for (int i = threadIdx.x; i < MF_RY * NQ; i += blockDim.x) {
        int tt = t2b + i / NQ;
        sp[i / NQ][i % NQ] = tt < Nt ? pts[(size_t)tt * NQ + i % NQ] : make_double4(0, 0, 0, 0);
    }
    if (threadIdx.x < MF_RY) {
        int tt = t2b + threadIdx.x;
        so[threadIdx.x] = tt < Nt ? origin[tt] : make_double4(0, 0, 0, 0);
    }
    if (tri_d) {
        for (int i = threadIdx.x; i < (32 + MF_RY) * 3; i += blockDim.x) {
            const int r = i / 3, l = i % 3;
            const int tt = r < 32 ? bx * 32 + r : t2b + (r - 32);
            const double4 v = tt < Nt ? tri_d[3 * (size_t)tt + l] : make_double4(0, 0, 0, 0);
            if (r < 32) sd1[r][l] = v;
            else sd2[r - 32][l] = v;
        }
    }
    __syncthreads();
    const int t2 = t2b + ty;
    if (t1 >= Nt || t2 >= Nt) return;
    if (sym && t1 > t2) return;
    if (skip[(size_t)t1 + (size_t)Nt * t2]) return;
    double4 p1[NQ];
#pragma unroll
    for (int p = 0; p < NQ; p++) p1[p] = pts[(size_t)t1 * NQ + p];
    const double4 o1 = origin[t1], o2 = so[ty];
    const double dox = o1.x - o2.x, doy = o1.y - o2.y, doz = o1.z - o2.z;
    double m[F][16];
#pragma unroll
    for (int f = 0; f < F; f++)
#pragma unroll
        for (int i = 0; i < 16; i++) m[f][i] = 0.0;
    constexpr double k4pi = 1.0 / (4.0 * kPi);
#pragma unroll 1
    for (int q = 0; q < NQ; q++) {
        const double4 pq = sp[ty][q];
        const double ax = dox - pq.x, ay = doy - pq.y, az = doz - pq.z;
        const double wq = pq.w * k4pi;
#pragma unroll
        for (int p = 0; p < NQ; p++) {
            const double dx = ax + p1[p].x, dy = ay + p1[p].y, dz = az + p1[p].z;
            const double R2 = fmax(dx * dx + dy * dy + dz * dz, 1e-30);
            const double rs = rsqrt(R2);
            const double R = R2 * rs;
            double inv = p1[p].w * wq * rs;
            double s0, c0, ss, cs;
            sincos(kr0 * R, &s0, &c0);
            const double x = dkr * R;
            if (fabs(x) <= 0.5) small_sincos(x, ss, cs);
            else sincos(x, &ss, &cs);
            if (ki0 != 0.0) inv *= exp(ki0 * R);
            double esr = cs, esi = -ss;   // e^{-j dk R}
            if (dki != 0.0) {
                const double e = exp(dki * R);
                esr *= e;
                esi *= e;
            }
            double gr = c0 * inv, gi = -s0 * inv;
            const double dd = p1[p].x * pq.x + p1[p].y * pq.y + p1[p].z * pq.z;
#pragma unroll
            for (int f = 0; f < F; f++) {
                m[f][0] += gr; m[f][1] += gi;
                m[f][2] += gr * p1[p].x; m[f][3] += gi * p1[p].x;
                m[f][4] += gr * p1[p].y; m[f][5] += gi * p1[p].y;
                m[f][6] += gr * p1[p].z; m[f][7] += gi * p1[p].z;
                m[f][8] += gr * pq.x; m[f][9] += gi * pq.x;
                m[f][10] += gr * pq.y; m[f][11] += gi * pq.y;
                m[f][12] += gr * pq.z; m[f][13] += gi * pq.z;
                m[f][14] += gr * dd; m[f][15] += gi * dd;
                if (f + 1 < F) {
                    const double nr = gr * esr - gi * esi;
                    gi = gr * esi + gi * esr;
                    gr = nr;
                }
            }
        }
    }
    const size_t slot = pair_slot(t1, t2, Nt, sym);
#pragma unroll
    for (int f = 0; f < F; f++) {
        if (tri_d) store_combo(ms.s[f], slot, sd1[tx], sd2[ty], m[f]);
        else store_mom(ms.s[f], slot, t1, t2, m[f]);
    }
}

// Generic point count (any Nq a prepack may carry).
__global__ void __launch_bounds__(256) k_regular_moments_any(
    int Nt, int Nq, bool sym, const double4 *__restrict__ origin, const double4 *__restrict__ pts,
    const uint8_t *__restrict__ skip, double kr, double ki, MomStore mom) {
    const int t1 = blockIdx.x * 32 + (threadIdx.x & 31);
    const int t2 = blockIdx.y * 8 + (threadIdx.x >> 5);
    if (t1 >= Nt || t2 >= Nt) return;
    if (sym && t1 > t2) return;
    if (skip[(size_t)t1 + (size_t)Nt * t2]) return;
    const double4 o1 = origin[t1], o2 = origin[t2];
    double m[16];
    for (int i = 0; i < 16; i++) m[i] = 0.0;
    for (int q = 0; q < Nq; q++) {
        const double4 pq = pts[(size_t)t2 * Nq + q];
        for (int p = 0; p < Nq; p++) {
            const double4 pp = pts[(size_t)t1 * Nq + p];
            const double dx = (o1.x - o2.x) + pp.x - pq.x, dy = (o1.y - o2.y) + pp.y - pq.y,
                         dz = (o1.z - o2.z) + pp.z - pq.z;
            double R = fmax(sqrt(dx * dx + dy * dy + dz * dz), 1e-15);
            double gr, gi;
            green(kr, ki, R, gr, gi);
            const double w = pp.w * pq.w;
            gr *= w;
            gi *= w;
            m[0] += gr; m[1] += gi;
            m[2] += gr * pp.x; m[3] += gi * pp.x; m[4] += gr * pp.y; m[5] += gi * pp.y;
            m[6] += gr * pp.z; m[7] += gi * pp.z;
            m[8] += gr * pq.x; m[9] += gi * pq.x; m[10] += gr * pq.y; m[11] += gi * pq.y;
            m[12] += gr * pq.z; m[13] += gi * pq.z;
            const double dd = pp.x * pq.x + pp.y * pq.y + pp.z * pq.z;
            m[14] += gr * dd; m[15] += gi * dd;
        }
    }
    store_mom(mom, pair_slot(t1, t2, Nt, sym), t1, t2, m);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// One point pair into the 16 moment accumulators.
__device__ __forceinline__ void acc_qpe(double *m, const double4 &pp, const double4 &pq, double gr, double gi) {
    const double w = pp.w * pq.w;
    gr *= w;
    gi *= w;
    m[0] += gr; m[1] += gi;
    m[2] += gr * pp.x; m[3] += gi * pp.x; m[4] += gr * pp.y; m[5] += gi * pp.y;
    m[6] += gr * pp.z; m[7] += gi * pp.z;
    m[8] += gr * pq.x; m[9] += gi * pq.x; m[10] += gr * pq.y; m[11] += gi * pq.y;
    m[12] += gr * pq.z; m[13] += gi * pq.z;
    const double dd = pp.x * pq.x + pp.y * pq.y + pp.z * pq.z;
    m[14] += gr * dd; m[15] += gi * dd;
}

// ---------------------------------------------------------------------------
// Near pairs (CPU_FAST.m:92-136; fastquad.cu:175-257): one warp per pair, the
// lanes share the point pairs of the subdivided rules; softening
// R = sqrt(R^2 + a^2), a = near_alpha * min(aeq(t1), aeq(t2)), then R >= 1e-15.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_near_moments(
    int Nt, bool sym, int n_pairs, const int2 *__restrict__ list, int P,
    const double4 *__restrict__ origin, const double4 *__restrict__ pts, const double *__restrict__ aeq,
    double near_alpha, double kr, double ki, MomStore mom) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= n_pairs) return;
    const int2 pr = list[warp];
    const int t1 = pr.x, t2 = pr.y;
    const double4 o1 = origin[t1], o2 = origin[t2];
    const double dox = o1.x - o2.x, doy = o1.y - o2.y, doz = o1.z - o2.z;
    const double a = near_alpha * fmin(aeq[t1], aeq[t2]);
    const double a2 = a * a;
    double m[16];
#pragma unroll
    for (int i = 0; i < 16; i++) m[i] = 0.0;
    const int total = P * P;
    for (int e = lane; e < total; e += 32) {
        const int p = e / P, q = e - p * P;
        const double4 pp = pts[(size_t)t1 * P + p];
        const double4 pq = pts[(size_t)t2 * P + q];
        const double dx = dox + pp.x - pq.x, dy = doy + pp.y - pq.y, dz = doz + pp.z - pq.z;
        double R = sqrt(dx * dx + dy * dy + dz * dz);
        R = sqrt(R * R + a2);
        R = fmax(R, 1e-15);
        double gr, gi;
        green(kr, ki, R, gr, gi);
        acc_qpe(m, pp, pq, gr, gi);
    }
#pragma unroll
    for (int i = 0; i < 16; i++) m[i] = warp_sum(m[i]);
    if (lane == 0) store_mom(mom, pair_slot(t1, t2, Nt, sym), t1, t2, m);
}

// ---------------------------------------------------------------------------
// Self pairs (CPU_FAST.m:139-183; fastquad.cu:260-345): one warp per
// triangle; softening R = sqrt(R^2 + aS(p)^2) only between points of the same
// sub-triangle, R = max(R, 1e-15) otherwise.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_self_moments(
    int Nt, bool sym, int P, int Nq2, const double4 *__restrict__ pts, const double *__restrict__ self_a,
    int NsS, double kr, double ki, MomStore mom) {
    const int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (t >= Nt) return;
    double m[16];
#pragma unroll
    for (int i = 0; i < 16; i++) m[i] = 0.0;
    const int total = P * P;
    for (int e = lane; e < total; e += 32) {
        const int p = e / P, q = e - p * P;
        const double4 pp = pts[(size_t)t * P + p];
        const double4 pq = pts[(size_t)t * P + q];
        const double dx = pp.x - pq.x, dy = pp.y - pq.y, dz = pp.z - pq.z;
        double R = sqrt(dx * dx + dy * dy + dz * dz);
        const int sp = p / Nq2, sq = q / Nq2;
        if (sp == sq) {
            const double aS = self_a[(size_t)t * NsS + sp];
            R = sqrt(R * R + aS * aS);
        } else {
            R = fmax(R, 1e-15);
        }
        double gr, gi;
        green(kr, ki, R, gr, gi);
        acc_qpe(m, pp, pq, gr, gi);
    }
#pragma unroll
    for (int i = 0; i < 16; i++) m[i] = warp_sum(m[i]);
    if (lane == 0) store_mom(mom, pair_slot(t, t, Nt, sym), t, t, m);
}

// Near and self pairs of F equally spaced frequencies in one launch (the
// reference scheme's subdivided rules): one warp per pair as in
// k_near_moments / k_self_moments, each point pair's R, 1/(4 pi R) and phase
// shared by the F frequencies as in k_regular_moments_mf.  Two warps per CTA:
// at up to 252 registers an SM holds eight warps either way, and small CTAs
// free their slots as soon as their own pairs are done.
template <int F>
__device__ __forceinline__ void acc_qpe_mf(double (&m)[F][16], const double4 &pp, const double4 &pq, double R2,
                                           double kr0, double ki0, double dkr, double dki) {
    R2 = fmax(R2, 1e-30);   // R >= 1e-15
    const double rs = rsqrt(R2);
    const double R = R2 * rs;
    double inv = pp.w * pq.w * (1.0 / (4.0 * kPi)) * rs;
    double s0, c0, ss, cs;
    sincos(kr0 * R, &s0, &c0);
    const double x = dkr * R;
    if (fabs(x) <= 0.5) small_sincos(x, ss, cs);
    else sincos(x, &ss, &cs);
    if (ki0 != 0.0) inv *= exp(ki0 * R);
    double esr = cs, esi = -ss;   // e^{-j dk R}
    if (dki != 0.0) {
        const double e = exp(dki * R);
        esr *= e;
        esi *= e;
    }
    double gr = c0 * inv, gi = -s0 * inv;
    const double dd = pp.x * pq.x + pp.y * pq.y + pp.z * pq.z;
#pragma unroll
    for (int f = 0; f < F; f++) {
        m[f][0] += gr; m[f][1] += gi;
        m[f][2] += gr * pp.x; m[f][3] += gi * pp.x;
        m[f][4] += gr * pp.y; m[f][5] += gi * pp.y;
        m[f][6] += gr * pp.z; m[f][7] += gi * pp.z;
        m[f][8] += gr * pq.x; m[f][9] += gi * pq.x;
        m[f][10] += gr * pq.y; m[f][11] += gi * pq.y;
        m[f][12] += gr * pq.z; m[f][13] += gi * pq.z;
        m[f][14] += gr * dd; m[f][15] += gi * dd;
        if (f + 1 < F) {
            const double nr = gr * esr - gi * esi;
            gi = gr * esi + gi * esr;
            gr = nr;
        }
    }
}

template <int F>
__device__ __forceinline__ void warp_store_mf(double (&m)[F][16], int lane, const MomStores &ms, size_t slot, int t1,
                                              int t2) {
#pragma unroll
    for (int f = 0; f < F; f++)
#pragma unroll
        for (int i = 0; i < 16; i++) m[f][i] = warp_sum(m[f][i]);
    if (lane == 0)
#pragma unroll
        for (int f = 0; f < F; f++) store_mom(ms.s[f], slot, t1, t2, m[f]);
}

template <int F>
__global__ void __launch_bounds__(64) k_near_moments_mf(
    int Nt, bool sym, int n_pairs, const int2 *__restrict__ list, int P, const double4 *__restrict__ origin,
    const double4 *__restrict__ pts, const double *__restrict__ aeq, double near_alpha, double kr0, double ki0,
    double dkr, double dki, MomStores ms) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= n_pairs) return;
    const int2 pr = list[warp];
    const int t1 = pr.x, t2 = pr.y;
    const double4 o1 = origin[t1], o2 = origin[t2];
    const double dox = o1.x - o2.x, doy = o1.y - o2.y, doz = o1.z - o2.z;
    const double a = near_alpha * fmin(aeq[t1], aeq[t2]);
    const double a2 = a * a;
    double m[F][16];
#pragma unroll
    for (int f = 0; f < F; f++)
#pragma unroll
        for (int i = 0; i < 16; i++) m[f][i] = 0.0;
    const int total = P * P;
    for (int e = lane; e < total; e += 32) {
        const int p = e / P, q = e - p * P;
        const double4 pp = pts[(size_t)t1 * P + p];
        const double4 pq = pts[(size_t)t2 * P + q];
        const double dx = dox + pp.x - pq.x, dy = doy + pp.y - pq.y, dz = doz + pp.z - pq.z;
        acc_qpe_mf<F>(m, pp, pq, dx * dx + dy * dy + dz * dz + a2, kr0, ki0, dkr, dki);
    }
    warp_store_mf<F>(m, lane, ms, pair_slot(t1, t2, Nt, sym), t1, t2);
}

template <int F>
__global__ void __launch_bounds__(64) k_self_moments_mf(int Nt, bool sym, int P, int Nq2,
                                                         const double4 *__restrict__ pts,
                                                         const double *__restrict__ self_a, int NsS, double kr0,
                                                         double ki0, double dkr, double dki, MomStores ms) {
    const int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (t >= Nt) return;
    double m[F][16];
#pragma unroll
    for (int f = 0; f < F; f++)
#pragma unroll
        for (int i = 0; i < 16; i++) m[f][i] = 0.0;
    const int total = P * P;
    for (int e = lane; e < total; e += 32) {
        const int p = e / P, q = e - p * P;
        const double4 pp = pts[(size_t)t * P + p];
        const double4 pq = pts[(size_t)t * P + q];
        const double dx = pp.x - pq.x, dy = pp.y - pq.y, dz = pp.z - pq.z;
        double R2 = dx * dx + dy * dy + dz * dz;
        const int sp = p / Nq2, sq = q / Nq2;
        if (sp == sq) {
            const double aS = self_a[(size_t)t * NsS + sp];
            R2 += aS * aS;
        }
        acc_qpe_mf<F>(m, pp, pq, R2, kr0, ki0, dkr, dki);
    }
    warp_store_mf<F>(m, lane, ms, pair_slot(t, t, Nt, sym), t, t);
}

// ---------------------------------------------------------------------------
// Extraction scheme (no reference counterpart): on self and vertex-adjacent
// pairs G = 1/(4 pi R) + (exp(-jkR) - 1)/(4 pi R).  The static part is
// integrated analytically over the inner triangle (potential integrals of
// Wilton et al. 1984 / Graglia 1993) at every outer rule point, the smooth
// part with the rule on both triangles.  One warp per pair (t1 <= t2).
// ---------------------------------------------------------------------------
// I0 = int_T 1/R dS', J = int_T (r' - r)/R dS' for triangle (a0, a1, a2).
__device__ void potential_integrals(const double3 a0, const double3 a1, const double3 a2, const double3 r,
                                    double &I0, double3 &J) {
    const double3 A[3] = {a0, a1, a2};
    double3 n = make_double3((a1.y - a0.y) * (a2.z - a0.z) - (a1.z - a0.z) * (a2.y - a0.y),
                             (a1.z - a0.z) * (a2.x - a0.x) - (a1.x - a0.x) * (a2.z - a0.z),
                             (a1.x - a0.x) * (a2.y - a0.y) - (a1.y - a0.y) * (a2.x - a0.x));
    const double nn = sqrt(n.x * n.x + n.y * n.y + n.z * n.z);
    n.x /= nn; n.y /= nn; n.z /= nn;
    const double d = n.x * (r.x - a0.x) + n.y * (r.y - a0.y) + n.z * (r.z - a0.z);
    const double ad = fabs(d);
    const double3 rho = make_double3(r.x - d * n.x, r.y - d * n.y, r.z - d * n.z);
    double s0 = 0.0, vx = 0.0, vy = 0.0, vz = 0.0;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const double3 p = A[i], q = A[(i + 1) % 3];
        double3 l = make_double3(q.x - p.x, q.y - p.y, q.z - p.z);
        const double ll = sqrt(l.x * l.x + l.y * l.y + l.z * l.z);
        l.x /= ll; l.y /= ll; l.z /= ll;
        const double3 u = make_double3(l.y * n.z - l.z * n.y, l.z * n.x - l.x * n.z, l.x * n.y - l.y * n.x);
        const double P0 = (p.x - rho.x) * u.x + (p.y - rho.y) * u.y + (p.z - rho.z) * u.z;
        const double lp = (q.x - rho.x) * l.x + (q.y - rho.y) * l.y + (q.z - rho.z) * l.z;
        const double lm = (p.x - rho.x) * l.x + (p.y - rho.y) * l.y + (p.z - rho.z) * l.z;
        const double R02 = P0 * P0 + d * d;
        const double Rp = sqrt(R02 + lp * lp), Rm = sqrt(R02 + lm * lm);
        double f;
        if (R02 < 1e-30 * (lp * lp + lm * lm)) {
            f = 0.0;   // point on the edge line: the terms vanish
        } else {
            // f = log((Rp + lp)/(Rm + lm)); R + l = R02/(R - l) where l < 0 avoids the cancellation
            const double np_ = lp >= 0.0 ? Rp + lp : R02 / (Rp - lp);
            const double nm_ = lm >= 0.0 ? Rm + lm : R02 / (Rm - lm);
            f = log(np_ / nm_);
        }
        double beta = 0.0;
        if (ad > 0.0) beta = atan(P0 * lp / (R02 + ad * Rp)) - atan(P0 * lm / (R02 + ad * Rm));
        s0 += P0 * f - ad * beta;
        const double t = 0.5 * (R02 * f + lp * Rp - lm * Rm);
        vx += u.x * t; vy += u.y * t; vz += u.z * t;
    }
    I0 = s0;
    J = make_double3(vx - d * n.x * s0, vy - d * n.y * s0, vz - d * n.z * s0);
}

// (exp(-jkR) - 1)/(4 pi R) without cancellation; -jk/(4 pi) at R = 0
__device__ __forceinline__ void smooth_green(double kr, double ki, double R, double &gr, double &gi) {
    if (R == 0.0) {
        gr = ki / (4.0 * kPi);
        gi = -kr / (4.0 * kPi);
        return;
    }
    double s, c, sh, ch;
    sincos(kr * R, &s, &c);
    sincos(0.5 * kr * R, &sh, &ch);
    const double em = expm1(ki * R);
    const double inv = 1.0 / (4.0 * kPi * R);
    gr = (em * c - 2.0 * sh * sh) * inv;
    gi = -(1.0 + em) * s * inv;
}

__global__ void __launch_bounds__(256) k_singular_moments(
    int Nt, int n_pairs, const int2 *__restrict__ list, int NQ, const double4 *__restrict__ origin,
    const double4 *__restrict__ pts, const double4 *__restrict__ vtx, double kr, double ki,
    MomStore mom) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= n_pairs) return;
    const int2 pr = list[warp];
    const int t1 = pr.x, t2 = pr.y;   // t1 <= t2: outer t1, inner t2
    const double4 o1 = origin[t1], o2 = origin[t2];
    const double dox = o1.x - o2.x, doy = o1.y - o2.y, doz = o1.z - o2.z;
    double m[16];
#pragma unroll
    for (int i = 0; i < 16; i++) m[i] = 0.0;
    // static part: outer point p on t1, analytic over t2 (coordinates relative to o2)
    if (lane < NQ) {
        const double4 pp = pts[(size_t)t1 * NQ + lane];
        const double3 r = make_double3(pp.x + dox, pp.y + doy, pp.z + doz);
        const double4 v0 = vtx[3 * (size_t)t2], v1 = vtx[3 * (size_t)t2 + 1], v2 = vtx[3 * (size_t)t2 + 2];
        double I0;
        double3 J;
        potential_integrals(make_double3(v0.x, v0.y, v0.z), make_double3(v1.x, v1.y, v1.z),
                            make_double3(v2.x, v2.y, v2.z), r, I0, J);
        // int rho' / R = J + (r - o2) I0   (rho' = r' - o2)
        const double sx = J.x + r.x * I0, sy = J.y + r.y * I0, sz = J.z + r.z * I0;
        const double w = pp.w / (4.0 * kPi);
        m[0] += w * I0;
        m[2] += w * I0 * pp.x; m[4] += w * I0 * pp.y; m[6] += w * I0 * pp.z;
        m[8] += w * sx; m[10] += w * sy; m[12] += w * sz;
        m[14] += w * (pp.x * sx + pp.y * sy + pp.z * sz);
    }
    // smooth part with the rule on both triangles
    for (int e = lane; e < NQ * NQ; e += 32) {
        const int p = e / NQ, q = e - p * NQ;
        const double4 pp = pts[(size_t)t1 * NQ + p];
        const double4 pq = pts[(size_t)t2 * NQ + q];
        const double dx = dox + pp.x - pq.x, dy = doy + pp.y - pq.y, dz = doz + pp.z - pq.z;
        const double R = sqrt(dx * dx + dy * dy + dz * dz);
        double gr, gi;
        smooth_green(kr, ki, R, gr, gi);
        acc_qpe(m, pp, pq, gr, gi);
    }
#pragma unroll
    for (int i = 0; i < 16; i++) m[i] = warp_sum(m[i]);
    if (t1 == t2) {
        // self pair: numeric-outer / analytic-inner is not symmetric in the two
        // sides; the mean of both orders (S1, S2 -> their average) keeps Z symmetric
#pragma unroll
        for (int i = 2; i < 8; i++) {
            const double s = 0.5 * (m[i] + m[i + 6]);
            m[i] = s;
            m[i + 6] = s;
        }
    }
    if (lane == 0) store_mom(mom, pair_slot(t1, t2, Nt, true), t1, t2, m);
}

// ---------------------------------------------------------------------------
// Gather: Z(m,n) = sum over the 4 triangle pairs of alpha Ivec + beta Isca,
// in the reference's (im, in) order (kernel_Z_fastquad, fastquad.cu:373-409).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 z_entry(int m, int n, int Ne, int Nt, bool sym, const int *__restrict__ etri,
                                           const double4 *__restrict__ ecd, const MomStore mom,
                                           double alr, double ali, double ber, double bei) {
    double zr = 0.0, zi = 0.0;
#pragma unroll
    for (int a = 0; a < 2; a++) {
        const int t1 = etri[a * Ne + m];
        if (t1 < 0) continue;
        const double4 dm = ecd[a * Ne + m];
#pragma unroll
        for (int b = 0; b < 2; b++) {
            const int t2 = etri[b * Ne + n];
            if (t2 < 0) continue;
            const double4 dn = ecd[b * Ne + n];
            const double2 *s = mom.p + pair_slot(t1, t2, Nt, sym);
            const size_t q = mom.stride;
            const double2 S0 = __ldg(s), S3 = __ldg(s + 7 * q);
            double2 S1x = __ldg(s + q), S1y = __ldg(s + 2 * q), S1z = __ldg(s + 3 * q), S2x = __ldg(s + 4 * q),
                    S2y = __ldg(s + 5 * q), S2z = __ldg(s + 6 * q);
            if (sym && t1 > t2) {  // stored for (t2, t1): swap the one-sided moments
                double2 tx = S1x, ty = S1y, tz = S1z;
                S1x = S2x; S1y = S2y; S1z = S2z;
                S2x = tx; S2y = ty; S2z = tz;
            }
            const double dd = dm.x * dn.x + dm.y * dn.y + dm.z * dn.z;
            const double ivr = S3.x - (dn.x * S1x.x + dn.y * S1y.x + dn.z * S1z.x)
                               - (dm.x * S2x.x + dm.y * S2y.x + dm.z * S2z.x) + dd * S0.x;
            const double ivi = S3.y - (dn.x * S1x.y + dn.y * S1y.y + dn.z * S1z.y)
                               - (dm.x * S2x.y + dm.y * S2y.y + dm.z * S2z.y) + dd * S0.y;
            const double cc = dm.w * dn.w;
            const double Ivr = cc * ivr, Ivi = cc * ivi;
            const double Isr = 4.0 * cc * S0.x, Isi = 4.0 * cc * S0.y;
            zr += (alr * Ivr - ali * Ivi) + (ber * Isr - bei * Isi);
            zi += (alr * Ivi + ali * Ivr) + (ber * Isi + bei * Isr);
        }
    }
    return make_double2(zr, zi);
}

// The same sum from the edge-combination form: etl[side][e] = 4 t + slot of
// the RWG side (-1: none), ec[side][e] its coefficient c.
__device__ __forceinline__ double2 z_entry_combo(int m, int n, int Ne, int Nt, bool sym, const int *__restrict__ etl,
                                                 const double *__restrict__ ec, const MomStore mom) {
    double zr = 0.0, zi = 0.0;
#pragma unroll
    for (int a = 0; a < 2; a++) {
        const int tm = etl[a * Ne + m];
        if (tm < 0) continue;
        const double cm = ec[a * Ne + m];
#pragma unroll
        for (int b = 0; b < 2; b++) {
            const int tn = etl[b * Ne + n];
            if (tn < 0) continue;
            const int t1 = tm >> 2, l1 = tm & 3, t2 = tn >> 2, l2 = tn & 3;
            // stored for (t2, t1) when t1 > t2 in the symmetric regime: the
            // integrand is symmetric, so the value sits at the swapped slots
            const bool sw = sym && t1 > t2;
            const int comp = sw ? 3 * l2 + l1 : 3 * l1 + l2;
            const double2 q = __ldg(mom.p + (size_t)comp * mom.stride + pair_slot(t1, t2, Nt, sym));
            const double cc = cm * ec[b * Ne + n];
            zr += cc * q.x;
            zi += cc * q.y;
        }
    }
    return make_double2(zr, zi);
}

struct EdgeData {
    const int *etri;      // triangle per RWG side (eight-moment form)
    const double4 *ecd;   // free vertex - origin, c
    const int *etl;       // 4 t + slot per RWG side (edge-combination form)
    const double *ec;     // c per RWG side
};

template <bool COMBO>
__device__ __forceinline__ double2 z_any(int m, int n, int Ne, int Nt, bool sym, const EdgeData &E,
                                         const MomStore &mom) {
    if (COMBO) return z_entry_combo(m, n, Ne, Nt, sym, E.etl, E.ec, mom);
    return z_entry(m, n, Ne, Nt, sym, E.etri, E.ecd, mom, mom.alr, mom.ali, mom.ber, mom.bei);
}

// Thread per entry, m fastest (column-major Z, coalesced stores).
template <bool COMBO>
__global__ void __launch_bounds__(256) k_gather_z(int Ne, int Nt, bool sym, const EdgeData E, const MomStore mom,
                                                  double2 *__restrict__ Z) {
    const int m = blockIdx.x * 64 + (threadIdx.x & 63);
    const int n = blockIdx.y * 4 + (threadIdx.x >> 6);
    if (m >= Ne || n >= Ne) return;
    Z[(size_t)m + (size_t)Ne * n] = z_any<COMBO>(m, n, Ne, Nt, sym, E, mom);
}

// Symmetric Z (symmetric pair regimes): only 32x32 tiles with bm <= bn are
// evaluated; an off-diagonal tile is also stored transposed through shared
// memory, so Z(n,m) is a bit-exact copy of Z(m,n).
// With pr set, the tile is also written as the complex64 working matrix of
// the mixed solver: FP32 planes re = pr[m * ld + n], im = pr[(Ne + m) * ld + n]
// (row-major, both triangles), coalesced through the same shared-memory tile.
template <bool COMBO>
__global__ void __launch_bounds__(256) k_gather_z_sym(int Ne, int Nt, const EdgeData E, const MomStore mom,
                                                      double2 *__restrict__ Z, float *__restrict__ pr, int ld) {
    const int bm = blockIdx.x, bn = blockIdx.y;
    if (bm > bn) return;
    __shared__ double2 tile[32][33];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int m = bm * 32 + tx;
    for (int j = ty; j < 32; j += 8) {
        const int n = bn * 32 + j;
        double2 z = make_double2(0.0, 0.0);
        if (m < Ne && n < Ne) {
            z = z_any<COMBO>(m, n, Ne, Nt, true, E, mom);
            Z[(size_t)m + (size_t)Ne * n] = z;
        }
        tile[j][tx] = z;
    }
    if (bm == bn && !pr) return;
    __syncthreads();
    if (pr) {
        float *pi = pr + (size_t)ld * Ne;
        // the L D L^T factorization reads the lower triangle of the planes
        // only (it writes the upper one itself): row m = bm * 32 + j,
        // columns n = bn * 32 + tx on the diagonal tiles
        if (bm == bn)
            for (int j = ty; j < 32; j += 8) {
                const int mm = bm * 32 + j, nn = bn * 32 + tx;
                if (mm < Ne && nn < Ne) {
                    const double2 v = tile[tx][j];
                    pr[(size_t)mm * ld + nn] = (float)v.x;
                    pi[(size_t)mm * ld + nn] = (float)v.y;
                }
            }
        if (bm != bn)   // row n = bn * 32 + j, columns m = bm * 32 + tx: Z(n, m) = Z(m, n)
            for (int j = ty; j < 32; j += 8) {
                const int nn = bn * 32 + j, mm = bm * 32 + tx;
                if (mm < Ne && nn < Ne) {
                    const double2 v = tile[j][tx];
                    pr[(size_t)nn * ld + mm] = (float)v.x;
                    pi[(size_t)nn * ld + mm] = (float)v.y;
                }
            }
    }
    if (bm == bn) return;
    // with the planes (the mixed solver), Z's lower triangle is written only
    // inside the 128 x 128 diagonal blocks that the symmetric GMRES product
    // reads in full; efie_z_mirror completes it for the paths that need all of Z
    if (pr && bm / 4 != bn / 4) return;
    for (int j = ty; j < 32; j += 8) {
        const int mm = bm * 32 + j, nn = bn * 32 + tx;
        if (mm < Ne && nn < Ne) Z[(size_t)nn + (size_t)Ne * mm] = tile[tx][j];
    }
}

// Z(n, m) = Z(m, n) on the 32 x 32 tiles that k_gather_z_sym leaves out with
// the planes (upper tile (bm, bn), bm < bn, in different 128-blocks)
__global__ void __launch_bounds__(256) k_z_mirror(int Ne, double2 *__restrict__ Z) {
    const int bm = blockIdx.x, bn = blockIdx.y;
    if (bm >= bn || bm / 4 == bn / 4) return;
    __shared__ double2 tile[32][33];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int j = ty; j < 32; j += 8) {
        const int m = bm * 32 + tx, n = bn * 32 + j;
        if (m < Ne && n < Ne) tile[j][tx] = Z[(size_t)m + (size_t)Ne * n];
    }
    __syncthreads();
    for (int j = ty; j < 32; j += 8) {
        const int mm = bm * 32 + j, nn = bn * 32 + tx;
        if (mm < Ne && nn < Ne) Z[(size_t)nn + (size_t)Ne * mm] = tile[tx][j];
    }
}

// ---------------------------------------------------------------------------
// Centroid (one point, weight = area) assembly: kernel_Z_centroid of
// gassemble_ZV_EFIE_RWG_DIFF_GPU_FAST.cu:49-106 with the host side data of
// :221-299.  side[2*Ne] = {pos.xyz, f.xyz, div, w, t(1-based, as double)}.
// ---------------------------------------------------------------------------
struct Side {
    double px, py, pz, fx, fy, fz, div, w, t, pad;
};

__global__ void __launch_bounds__(256) k_centroid_z(int Ne, const Side *__restrict__ side,
                                                    const double *__restrict__ asoft, double kr, double ki,
                                                    double alr, double ali, double ber, double bei,
                                                    double2 *__restrict__ Z) {
    const int m = blockIdx.x * 64 + (threadIdx.x & 63);
    const int n = blockIdx.y * 4 + (threadIdx.x >> 6);
    if (m >= Ne || n >= Ne) return;
    double zr = 0.0, zi = 0.0;
    for (int sa = 0; sa < 2; sa++) {
        const Side A = side[2 * m + sa];
        if (A.w == 0.0 || A.t == 0.0) continue;
        for (int sb = 0; sb < 2; sb++) {
            const Side B = side[2 * n + sb];
            if (B.w == 0.0 || B.t == 0.0) continue;
            const double dx = A.px - B.px, dy = A.py - B.py, dz = A.pz - B.pz;
            double R = sqrt(dx * dx + dy * dy + dz * dz);
            if (A.t == B.t) {
                const double a = asoft[(int)A.t - 1];
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

// The pair mask (1 = near, adjacent or self: not a regular pair) from the
// pair list, on a zeroed mask: entry (t1, t2) and, for a symmetric list, (t2, t1).
__global__ void k_mask_pairs(int Nt, int n, const int2 *__restrict__ list, bool both, uint8_t *__restrict__ mask) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int2 pr = list[i];
    mask[(size_t)pr.x + (size_t)Nt * pr.y] = 1;
    if (both) mask[(size_t)pr.y + (size_t)Nt * pr.x] = 1;
}

__global__ void k_mask_self(int Nt, uint8_t *__restrict__ mask) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < Nt) mask[(size_t)t * (Nt + 1)] = 1;
}

}  // namespace

Physics efie_physics_k(efie_c128 k, double omega, double mu, efie_c128 eps) {
    Physics p;
    p.kr = k.re;
    p.ki = k.im;
    // alpha = j w mu ; beta = 1/(j w eps)  (ggassemble.cu:678-686)
    p.alr = 0.0;
    p.ali = omega * mu;
    const double dr = -omega * eps.im, di = omega * eps.re, d2 = dr * dr + di * di;
    p.ber = dr / d2;
    p.bei = -di / d2;
    return p;
}

Physics efie_physics(double freq, double mu, efie_c128 eps) {
    // patch_sweep_fastquad_cuda.cu:714-743: principal sqrt by the polar form
    const double omega = 2.0 * kPi * freq;
    const double ar = mu * eps.re, ai = mu * eps.im;
    const double r = std::sqrt(ar * ar + ai * ai), ang = std::atan2(ai, ar);
    const double sr = std::sqrt(r), half = 0.5 * ang;
    efie_c128 k = {omega * (sr * std::cos(half)), omega * (sr * std::sin(half))};
    return efie_physics_k(k, omega, mu, eps);
}

// Host-side repacking of the boundary arrays into the device layout.
efie_status efie_geom_upload(efie_ctx *ctx, const efie_mesh *mesh, const efie_prepack *pre, int scheme,
                             int rule_order, GeomDev &g, const efie_precompute_opts *popts) {
    const int Ne = mesh->Ne, Nt = mesh->Nt, Nv = mesh->Nv;
    g.Ne = Ne;
    g.Nt = Nt;
    g.scheme = scheme;
    g.near_alpha = pre ? pre->near_alpha : 0.0;
    if (scheme == EFIE_SCHEME_REF && !pre && !popts)
        return efie_fail(EFIE_ERR_PREPACK, "the reference scheme needs a prepack or precompute options");
    // origins: triangle centroids from V/F
    std::vector<double4> origin(Nt);
    for (int t = 0; t < Nt; t++) {
        double c[3] = {0, 0, 0};
        for (int j = 0; j < 3; j++) {
            const int v = mesh->F[t + (size_t)j * Nt] - 1;
            for (int k = 0; k < 3; k++) c[k] += mesh->V[v + (size_t)k * Nv];
        }
        origin[t] = make_double4(c[0] / 3.0, c[1] / 3.0, c[2] / 3.0, 0.0);
    }
    auto up = [&](DevBuf &b, const void *src, size_t bytes) -> efie_status {
        EFIE_TRY(b.reserve(bytes));
        EFIE_CUDA(cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
        return EFIE_OK;
    };
    // edges: per side triangle (0-based, -1 = none), delta = v - o, c
    std::vector<int> etri(2 * (size_t)Ne);
    std::vector<double4> ecd(2 * (size_t)Ne);
    for (int e = 0; e < Ne; e++) {
        const int tp = mesh->plusTri[e], tm = mesh->minusTri[e];
        const double l = mesh->len[e];
        for (int sd = 0; sd < 2; sd++) {
            int t = sd == 0 ? tp : tm;
            // rwg_eval_point picks the plus formula whenever t == plusTri
            // (fastquad.cu:82-95), also for a degenerate edge with tp == tm.
            const bool plus = (sd == 0) || (tm == tp);
            double c;
            const double *v = plus ? mesh->rp : mesh->rm;
            if (plus) c = (double)mesh->plusSign[e] * (l / (2.0 * mesh->Ap[e]));
            else c = -((double)mesh->minusSign[e] * (l / (2.0 * mesh->Am[e])));
            if (t <= 0) {
                etri[sd * (size_t)Ne + e] = -1;
                ecd[sd * (size_t)Ne + e] = make_double4(0, 0, 0, 0);
                continue;
            }
            const double4 o = origin[t - 1];
            etri[sd * (size_t)Ne + e] = t - 1;
            ecd[sd * (size_t)Ne + e] = make_double4(v[e] - o.x, v[e + Ne] - o.y, v[e + 2 * (size_t)Ne] - o.z, c);
        }
    }
    EFIE_TRY(up(g.origin, origin.data(), sizeof(double4) * Nt));
    EFIE_TRY(up(g.edge_tri, etri.data(), sizeof(int) * etri.size()));
    EFIE_TRY(up(g.edge_cd, ecd.data(), sizeof(double4) * ecd.size()));
    // free-vertex slots of the edge-combination moments: the distinct vectors
    // v - o of the RWG sides on each triangle (bitwise), at most three for a
    // mesh whose RWG free vertices are vertices of their triangles; otherwise
    // the eight-moment form is kept
    {
        std::vector<double4> trid(3 * (size_t)Nt, make_double4(0, 0, 0, 0));
        std::vector<int> nslot(Nt, 0), etl(2 * (size_t)Ne, -1);
        std::vector<double> ec(2 * (size_t)Ne, 0.0);
        bool combo = true;
        for (size_t i = 0; i < 2 * (size_t)Ne && combo; i++) {
            const int t = etri[i];
            if (t < 0) continue;
            const double4 d = ecd[i];
            int l = 0;
            while (l < nslot[t] && !(trid[3 * (size_t)t + l].x == d.x && trid[3 * (size_t)t + l].y == d.y &&
                                     trid[3 * (size_t)t + l].z == d.z))
                l++;
            if (l == nslot[t]) {
                if (l == 3) {
                    combo = false;
                    break;
                }
                trid[3 * (size_t)t + l] = make_double4(d.x, d.y, d.z, 0.0);
                nslot[t]++;
            }
            etl[i] = 4 * t + l;
            ec[i] = d.w;
        }
        g.combo = combo;
        if (combo) {
            EFIE_TRY(up(g.tri_d, trid.data(), sizeof(double4) * trid.size()));
            EFIE_TRY(up(g.edge_tl, etl.data(), sizeof(int) * etl.size()));
            EFIE_TRY(up(g.edge_c, ec.data(), sizeof(double) * ec.size()));
        }
    }

    // the pair list whose entries (and diagonal) the device mask marks
    std::vector<int2> list;
    bool mask_both = true;
    if (scheme == EFIE_SCHEME_REF && !pre) {
        // caches and near-pair list computed on the device from V/F (precompute.cu)
        EFIE_TRY(efie_geom_precompute_device(ctx, mesh, popts, g));
    } else if (scheme == EFIE_SCHEME_REF) {
        const int Nq = pre->Nq, Nq2 = pre->Nq2, NsS = pre->NsS, NsN = pre->NsN;
        g.Nq = Nq;
        g.Nq2 = Nq2;
        g.NsS = NsS;
        g.NsN = NsN;
        std::vector<double4> reg((size_t)Nt * Nq), nearp((size_t)Nt * NsN * Nq2), selfp((size_t)Nt * NsS * Nq2);
        for (int t = 0; t < Nt; t++) {
            const double4 o = origin[t];
            for (int i = 0; i < Nq; i++) {
                const double *r = pre->r_reg + i + (size_t)Nq * 3 * t;
                reg[(size_t)t * Nq + i] = make_double4(r[0] - o.x, r[Nq] - o.y, r[2 * Nq] - o.z,
                                                       pre->w_reg[i + (size_t)Nq * t]);
            }
            for (int p = 0; p < NsN; p++)
                for (int i = 0; i < Nq2; i++) {
                    const double *r = pre->near_r + i + (size_t)Nq2 * 3 * p + (size_t)Nq2 * 3 * NsN * t;
                    nearp[((size_t)t * NsN + p) * Nq2 + i] =
                        make_double4(r[0] - o.x, r[Nq2] - o.y, r[2 * Nq2] - o.z,
                                     pre->near_w[i + (size_t)Nq2 * p + (size_t)Nq2 * NsN * t]);
                }
            for (int p = 0; p < NsS; p++)
                for (int i = 0; i < Nq2; i++) {
                    const double *r = pre->self_r + i + (size_t)Nq2 * 3 * p + (size_t)Nq2 * 3 * NsS * t;
                    selfp[((size_t)t * NsS + p) * Nq2 + i] =
                        make_double4(r[0] - o.x, r[Nq2] - o.y, r[2 * Nq2] - o.z,
                                     pre->self_w[i + (size_t)Nq2 * p + (size_t)Nq2 * NsS * t]);
                }
        }
        EFIE_TRY(up(g.reg_pts, reg.data(), sizeof(double4) * reg.size()));
        EFIE_TRY(up(g.near_pts, nearp.data(), sizeof(double4) * nearp.size()));
        EFIE_TRY(up(g.self_pts, selfp.data(), sizeof(double4) * selfp.size()));
        EFIE_TRY(up(g.self_a, pre->self_a, sizeof(double) * (size_t)Nt * NsS));
        EFIE_TRY(up(g.aeq, pre->aeqTri, sizeof(double) * Nt));
        // near pairs (t1 != t2, nearMat nonzero) column by column, skipping
        // zero bytes eight at a time: nearMat is almost all zeros
        std::vector<int2> all;
        for (int t2 = 0; t2 < Nt; t2++) {
            const uint8_t *col = pre->nearMat + (size_t)Nt * t2;
            int t1 = 0;
            for (; t1 + 8 <= Nt; t1 += 8) {
                uint64_t w;
                std::memcpy(&w, col + t1, 8);
                if (!w) continue;
                for (int j = 0; j < 8; j++)
                    if (col[t1 + j] && t1 + j != t2) all.push_back(make_int2(t1 + j, t2));
            }
            for (; t1 < Nt; t1++)
                if (col[t1] && t1 != t2) all.push_back(make_int2(t1, t2));
        }
        // pair regimes; symmetric storage only if nearMat is symmetric: every
        // (t1, t2) of the list has its (t2, t1)
        std::vector<int64_t> keys(all.size());
        for (size_t i = 0; i < all.size(); i++) keys[i] = (int64_t)all[i].x * Nt + all[i].y;
        std::sort(keys.begin(), keys.end());
        bool sym = true;
        for (size_t i = 0; i < all.size() && sym; i++)
            sym = std::binary_search(keys.begin(), keys.end(), (int64_t)all[i].y * Nt + all[i].x);
        g.symmetric = sym;
        // the near list in column order (t1 < t2 when symmetric)
        for (const int2 &pr : all)
            if (!sym || pr.x < pr.y) list.push_back(pr);
        mask_both = sym;
        g.n_near = (int)list.size();
        EFIE_TRY(up(g.near_list, list.data(), sizeof(int2) * (list.empty() ? 1 : list.size())));
    } else if (scheme == EFIE_SCHEME_EXTRACT) {
        // rule points of every triangle from V/F (map_ref_to_vertices.m form), weights times 2A
        const int order = rule_order ? rule_order : EFIE_QUAD_DUNAVANT7;
        double qu[7], qv[7], qw[7];
        const int Nq = efie_quad_rule(order, qu, qv, qw);
        g.Nq = Nq;
        std::vector<double4> reg((size_t)Nt * Nq), vtx(3 * (size_t)Nt);
        for (int t = 0; t < Nt; t++) {
            double a[3][3];
            for (int j = 0; j < 3; j++) {
                const int v = mesh->F[t + (size_t)j * Nt] - 1;
                for (int k = 0; k < 3; k++) a[j][k] = mesh->V[v + (size_t)k * Nv];
            }
            const double4 o = origin[t];
            const double e1[3] = {a[1][0] - a[0][0], a[1][1] - a[0][1], a[1][2] - a[0][2]};
            const double e2[3] = {a[2][0] - a[0][0], a[2][1] - a[0][1], a[2][2] - a[0][2]};
            const double cx = e1[1] * e2[2] - e1[2] * e2[1], cy = e1[2] * e2[0] - e1[0] * e2[2],
                         cz = e1[0] * e2[1] - e1[1] * e2[0];
            const double a2 = std::sqrt(cx * cx + cy * cy + cz * cz);
            for (int i = 0; i < Nq; i++)
                reg[(size_t)t * Nq + i] = make_double4(a[0][0] + qu[i] * e1[0] + qv[i] * e2[0] - o.x,
                                                       a[0][1] + qu[i] * e1[1] + qv[i] * e2[1] - o.y,
                                                       a[0][2] + qu[i] * e1[2] + qv[i] * e2[2] - o.z, qw[i] * a2);
            for (int j = 0; j < 3; j++) vtx[3 * (size_t)t + j] = make_double4(a[j][0] - o.x, a[j][1] - o.y, a[j][2] - o.z, 0.0);
        }
        EFIE_TRY(up(g.reg_pts, reg.data(), sizeof(double4) * reg.size()));
        EFIE_TRY(up(g.tri_vtx, vtx.data(), sizeof(double4) * vtx.size()));
        // self and vertex-adjacent pairs (t1 <= t2) through a vertex -> triangles map
        std::vector<std::vector<int>> vt(Nv);
        for (int t = 0; t < Nt; t++)
            for (int j = 0; j < 3; j++) vt[mesh->F[t + (size_t)j * Nt] - 1].push_back(t);
        std::vector<int> seen(Nt, -1);
        for (int t1 = 0; t1 < Nt; t1++) {
            for (int j = 0; j < 3; j++)
                for (int t2 : vt[mesh->F[t1 + (size_t)j * Nt] - 1])
                    if (t2 >= t1 && seen[t2] != t1) {
                        seen[t2] = t1;
                        list.push_back(make_int2(t1, t2));
                    }
        }
        g.symmetric = true;
        g.n_adj = (int)list.size();
        g.n_near = 0;
        EFIE_TRY(up(g.adj_list, list.data(), sizeof(int2) * (list.empty() ? 1 : list.size())));
    } else {
        return efie_fail(EFIE_ERR_ARGS, "unknown scheme");
    }
    // the pair mask is built on the device from the list: zeros, the list's
    // entries (both orientations when symmetric), the diagonal
    {
        const size_t nn = (size_t)Nt * Nt;
        EFIE_TRY(g.near_mask.reserve(nn));
        EFIE_CUDA(cudaMemsetAsync(g.near_mask.p, 0, nn, ctx->stream));
        DevBuf &lst = scheme == EFIE_SCHEME_REF ? g.near_list : g.adj_list;
        const int n = scheme == EFIE_SCHEME_REF ? g.n_near : g.n_adj;
        if (n > 0)
            k_mask_pairs<<<(n + 255) / 256, 256, 0, ctx->stream>>>(Nt, n, lst.as<int2>(), mask_both,
                                                                   g.near_mask.as<uint8_t>());
        k_mask_self<<<(Nt + 255) / 256, 256, 0, ctx->stream>>>(Nt, g.near_mask.as<uint8_t>());
        EFIE_CUDA(cudaGetLastError());
    }
    g.npairs = g.symmetric ? (size_t)Nt * (Nt + 1) / 2 : (size_t)Nt * Nt;
    if (g.symmetric) {
        // the 32 x MF_RY tiles of the multi-frequency launches with t1 block <= t2 block
        std::vector<int2> tl;
        const int ntx = (Nt + 31) / 32, nty = (Nt + MF_RY - 1) / MF_RY;
        for (int by = 0; by < nty; by++)
            for (int bx = 0; bx < ntx && bx * 32 <= by * MF_RY + MF_RY - 1; bx++) tl.push_back(make_int2(bx, by));
        g.n_reg_tiles = (int)tl.size();
        EFIE_TRY(up(g.reg_tiles, tl.data(), sizeof(int2) * tl.size()));
    }
    // component planes of npairs (9 edge combinations or the 8 moments) for up
    // to four frequencies assembled together, within a quarter of free memory
    const size_t per = sizeof(double2) * (g.combo ? 9 : 8) * g.npairs;
    size_t freeb = 0, totalb = 0;
    g.mf = 1;
    if ((g.Nq == 3 || g.Nq == 7) && cudaMemGetInfo(&freeb, &totalb) == cudaSuccess)
        for (int f = 4; f >= 2; f--)
            if (f * per <= freeb / 4) {
                g.mf = f;
                break;
            }
    EFIE_TRY(g.moments.reserve(per * g.mf));
    return EFIE_OK;
}

namespace {

// the pair-value store of frequency slot j of the geometry's moment buffer
MomStore mom_store(const GeomDev &g, const Physics &ph, int j) {
    const size_t planes = g.combo ? 9 : 8;
    return MomStore{g.moments.as<double2>() + (size_t)j * planes * g.npairs, g.npairs,
                    g.combo ? g.tri_d.as<double4>() : nullptr, ph.alr, ph.ali, ph.ber, ph.bei};
}

double regular_pairs(const GeomDev &g) {
    // regular pairs evaluated: all pairs (or t1 <= t2) minus near/self ones
    const double all = g.symmetric ? 0.5 * (double)g.Nt * (g.Nt + 1) : (double)g.Nt * g.Nt;
    return g.scheme == EFIE_SCHEME_EXTRACT ? all - (double)g.n_adj : all - (double)g.n_near - (double)g.Nt;
}

template <int F>
void launch_regular_mf(const GeomDev &g, cudaStream_t s, const Physics *ph, const MomStores &ms) {
    // symmetric pairs: the tiles on or above the diagonal from the list
    const bool lst = g.symmetric && g.n_reg_tiles > 0;
    dim3 grid = lst ? dim3((unsigned)g.n_reg_tiles) : dim3((g.Nt + 31) / 32, (g.Nt + MF_RY - 1) / MF_RY);
    const int2 *tiles = lst ? g.reg_tiles.as<int2>() : nullptr;
    const double4 *org = g.origin.as<double4>(), *pts = g.reg_pts.as<double4>();
    const uint8_t *skip = g.near_mask.as<uint8_t>();
    const double dkr = (ph[F - 1].kr - ph[0].kr) / (F - 1), dki = (ph[F - 1].ki - ph[0].ki) / (F - 1);
    switch (g.Nq) {
    case 3:
        k_regular_moments_mf<3, F><<<grid, 32 * MF_RY, 0, s>>>(g.Nt, g.symmetric, tiles, org, pts, skip, ph[0].kr, ph[0].ki,
                                                        dkr, dki, ms);
        break;
    case 7:
        k_regular_moments_mf<7, F><<<grid, 32 * MF_RY, 0, s>>>(g.Nt, g.symmetric, tiles, org, pts, skip, ph[0].kr, ph[0].ki,
                                                        dkr, dki, ms);
        break;
    }
}

template <int F>
void launch_nearself_mf(const GeomDev &g, cudaStream_t s, const Physics *ph, const MomStores &ms, double &qpe,
                        int &nl) {
    const double dkr = (ph[F - 1].kr - ph[0].kr) / (F - 1), dki = (ph[F - 1].ki - ph[0].ki) / (F - 1);
    const double4 *org = g.origin.as<double4>();
    if (g.n_near > 0) {
        const int P = g.NsN * g.Nq2;
        k_near_moments_mf<F><<<(g.n_near + 1) / 2, 64, 0, s>>>(g.Nt, g.symmetric, g.n_near, g.near_list.as<int2>(),
                                                                P, org, g.near_pts.as<double4>(), g.aeq.as<double>(),
                                                                g.near_alpha, ph[0].kr, ph[0].ki, dkr, dki, ms);
        nl++;
        qpe += (double)g.n_near * P * P;
    }
    const int P = g.NsS * g.Nq2;
    k_self_moments_mf<F><<<(g.Nt + 1) / 2, 64, 0, s>>>(g.Nt, g.symmetric, P, g.Nq2, g.self_pts.as<double4>(),
                                                        g.self_a.as<double>(), g.NsS, ph[0].kr, ph[0].ki, dkr, dki,
                                                        ms);
    nl++;
    qpe += (double)g.Nt * P * P;
}

// k_f = k0 + f dk within 1e-12 |k_f| for f < n
bool equally_spaced(const Physics *ph, int n) {
    if (n < 2) return false;
    const double dkr = (ph[n - 1].kr - ph[0].kr) / (n - 1), dki = (ph[n - 1].ki - ph[0].ki) / (n - 1);
    for (int f = 1; f < n - 1; f++) {
        const double er = ph[0].kr + f * dkr - ph[f].kr, ei = ph[0].ki + f * dki - ph[f].ki;
        if (std::hypot(er, ei) > 1e-12 * std::hypot(ph[f].kr, ph[f].ki)) return false;
    }
    return true;
}

}  // namespace

efie_status efie_assemble_finish(efie_ctx *ctx, GeomDev &g, const Physics &ph, int j, void *Z, float *pr, int ld,
                                 bool nearself_done = false);

efie_status efie_assemble_device(efie_ctx *ctx, GeomDev &g, const Physics &ph, void *Z, float *pr, int ld) {
    cudaStream_t s = ctx->stream;
    KernelLog &log = ctx->log;
    const int Nt = g.Nt;
    const MomStore mom = mom_store(g, ph, 0);
    dim3 grid((Nt + 31) / 32, (Nt + 7) / 8);
    const double4 *org = g.origin.as<double4>(), *pts = g.reg_pts.as<double4>();
    const uint8_t *skip = g.near_mask.as<uint8_t>();
    const double n_regular = regular_pairs(g);
    size_t tok = log.begin(s);
    switch (g.Nq) {
    case 1: k_regular_moments<1><<<grid, 256, 0, s>>>(Nt, g.symmetric, org, pts, skip, ph.kr, ph.ki, mom); break;
    case 3: k_regular_moments<3><<<grid, 256, 0, s>>>(Nt, g.symmetric, org, pts, skip, ph.kr, ph.ki, mom); break;
    case 6: k_regular_moments<6><<<grid, 256, 0, s>>>(Nt, g.symmetric, org, pts, skip, ph.kr, ph.ki, mom); break;
    case 7: k_regular_moments<7><<<grid, 256, 0, s>>>(Nt, g.symmetric, org, pts, skip, ph.kr, ph.ki, mom); break;
    default:
        k_regular_moments_any<<<grid, 256, 0, s>>>(Nt, g.Nq, g.symmetric, org, pts, skip, ph.kr, ph.ki, mom);
    }
    EFIE_CUDA(cudaGetLastError());
    log.end(EFIE_K_QUAD, s, tok, n_regular * (double)g.Nq * g.Nq);
    return efie_assemble_finish(ctx, g, ph, 0, Z, pr, ld);
}

// Frequencies of a batch: equally spaced runs of up to g.mf frequencies share
// one regular-pair launch (the Nq = 3 and 7 rules), then each frequency's
// near/self or singular pairs and gather run on its own store.
efie_status efie_assemble_batch(efie_ctx *ctx, GeomDev &g, const Physics *ph, int nf, void *const *Z,
                                const PlanesOut *po) {
    if (po && !g.symmetric) return efie_fail(EFIE_ERR_ARGS, "complex64 planes need the symmetric gather");
    auto planes = [&](int f) { return po ? po->p + po->pstride * f : nullptr; };
    const int ld = po ? po->ld : 0;
    int f0 = 0;
    while (f0 < nf) {
        int n = std::min(g.mf, nf - f0);
        while (n > 1 && !equally_spaced(ph + f0, n)) n--;
        if (n < 2 || (g.Nq != 3 && g.Nq != 7)) {
            EFIE_TRY(efie_assemble_device(ctx, g, ph[f0], Z[f0], planes(f0), ld));
            f0++;
            continue;
        }
        MomStores ms{};
        for (int j = 0; j < n; j++) ms.s[j] = mom_store(g, ph[f0 + j], j);
        size_t tok = ctx->log.begin(ctx->stream);
        if (n == 2) launch_regular_mf<2>(g, ctx->stream, ph + f0, ms);
        else if (n == 3) launch_regular_mf<3>(g, ctx->stream, ph + f0, ms);
        else launch_regular_mf<4>(g, ctx->stream, ph + f0, ms);
        EFIE_CUDA(cudaGetLastError());
        ctx->log.end(EFIE_K_QUAD, ctx->stream, tok, n * regular_pairs(g) * (double)g.Nq * g.Nq);
        // the reference scheme's near and self pairs of the group, likewise
        const bool ns = g.scheme == EFIE_SCHEME_REF;
        if (ns) {
            tok = ctx->log.begin(ctx->stream);
            double qpe = 0;
            int nl = 0;
            if (n == 2) launch_nearself_mf<2>(g, ctx->stream, ph + f0, ms, qpe, nl);
            else if (n == 3) launch_nearself_mf<3>(g, ctx->stream, ph + f0, ms, qpe, nl);
            else launch_nearself_mf<4>(g, ctx->stream, ph + f0, ms, qpe, nl);
            EFIE_CUDA(cudaGetLastError());
            ctx->log.end(EFIE_K_NEARSELF, ctx->stream, tok, n * qpe, nl);
        }
        for (int j = 0; j < n; j++)
            EFIE_TRY(efie_assemble_finish(ctx, g, ph[f0 + j], j, Z[f0 + j], planes(f0 + j), ld, ns));
        f0 += n;
    }
    return EFIE_OK;
}

// Near/self (or singular) pairs of one frequency into store j, then its gather.
efie_status efie_assemble_finish(efie_ctx *ctx, GeomDev &g, const Physics &ph, int j, void *Z, float *pr, int ld,
                                 bool nearself_done) {
    cudaStream_t s = ctx->stream;
    KernelLog &log = ctx->log;
    const int Nt = g.Nt, Ne = g.Ne;
    const MomStore mom = mom_store(g, ph, j);
    const double4 *org = g.origin.as<double4>();
    size_t tok = log.begin(s);
    int nl = 0;
    double qpe = 0;
    if (nearself_done) {
    } else if (g.scheme == EFIE_SCHEME_EXTRACT) {
        k_singular_moments<<<(g.n_adj + 7) / 8, 256, 0, s>>>(Nt, g.n_adj, g.adj_list.as<int2>(), g.Nq, org,
                                                            g.reg_pts.as<double4>(), g.tri_vtx.as<double4>(), ph.kr,
                                                            ph.ki, mom);
        EFIE_CUDA(cudaGetLastError());
        log.end(EFIE_K_NEARSELF, s, tok, (double)g.n_adj * g.Nq * (g.Nq + 1), 1);
    } else {
    if (g.n_near > 0) {
        const int P = g.NsN * g.Nq2;
        k_near_moments<<<(g.n_near + 7) / 8, 256, 0, s>>>(Nt, g.symmetric, g.n_near, g.near_list.as<int2>(), P, org,
                                                        g.near_pts.as<double4>(), g.aeq.as<double>(), g.near_alpha,
                                                        ph.kr, ph.ki, mom);
        EFIE_CUDA(cudaGetLastError());
        nl++;
        qpe += (double)g.n_near * P * P;
    }
    {
        const int P = g.NsS * g.Nq2;
        k_self_moments<<<(Nt + 7) / 8, 256, 0, s>>>(Nt, g.symmetric, P, g.Nq2, g.self_pts.as<double4>(),
                                                   g.self_a.as<double>(), g.NsS, ph.kr, ph.ki, mom);
        EFIE_CUDA(cudaGetLastError());
        nl++;
        qpe += (double)Nt * P * P;
    }
    log.end(EFIE_K_NEARSELF, s, tok, qpe, nl);
    }
    tok = log.begin(s);
    const EdgeData E{g.edge_tri.as<int>(), g.edge_cd.as<double4>(), g.edge_tl.as<int>(), g.edge_c.as<double>()};
    double2 *Zd = static_cast<double2 *>(Z);
    if (g.symmetric) {
        dim3 gs((Ne + 31) / 32, (Ne + 31) / 32);
        if (g.combo) k_gather_z_sym<true><<<gs, 256, 0, s>>>(Ne, Nt, E, mom, Zd, pr, ld);
        else k_gather_z_sym<false><<<gs, 256, 0, s>>>(Ne, Nt, E, mom, Zd, pr, ld);
    } else {
        dim3 gg((Ne + 63) / 64, (Ne + 3) / 4);
        if (g.combo) k_gather_z<true><<<gg, 256, 0, s>>>(Ne, Nt, false, E, mom, Zd);
        else k_gather_z<false><<<gg, 256, 0, s>>>(Ne, Nt, false, E, mom, Zd);
    }
    EFIE_CUDA(cudaGetLastError());
    // algorithmic bytes: one read of every pair value, Z written once (with
    // the planes: Z's upper and the planes' lower triangle)
    log.end(EFIE_K_GATHER, s, tok,
            16.0 * (g.combo ? 9.0 : 8.0) * (double)g.npairs +
                (pr ? 12.0 * (double)Ne * (Ne + 1) : 16.0 * (double)Ne * Ne));
    return EFIE_OK;
}

efie_status efie_z_mirror(efie_ctx *ctx, void *Z, int Ne) {
    dim3 gs((Ne + 31) / 32, (Ne + 31) / 32);
    k_z_mirror<<<gs, 256, 0, ctx->stream>>>(Ne, static_cast<double2 *>(Z));
    EFIE_CUDA(cudaGetLastError());
    return EFIE_OK;
}

efie_status efie_assemble_centroid_device(efie_ctx *ctx, const efie_mesh *mesh, double selfAlpha, const Physics &ph,
                                          void *Z, DevBuf &scratch) {
    const int Ne = mesh->Ne, Nt = mesh->Nt, Nv = mesh->Nv;
    // gassemble.cu:221-299: centroids, areas, softening, side data (host, FP64)
    std::vector<double> cent(3 * (size_t)Nt), asoft(Nt);
    for (int t = 0; t < Nt; t++) {
        int id[3];
        for (int j = 0; j < 3; j++) {
            id[j] = mesh->F[t + (size_t)j * Nt] - 1;
            if (id[j] < 0 || id[j] >= Nv) return efie_fail(EFIE_ERR_F, "F has invalid indices.");
        }
        double r[3][3];
        for (int j = 0; j < 3; j++)
            for (int k = 0; k < 3; k++) r[j][k] = mesh->V[id[j] + (size_t)k * Nv];
        for (int k = 0; k < 3; k++) cent[3 * t + k] = (r[0][k] + r[1][k] + r[2][k]) / 3.0;
        const double e1[3] = {r[1][0] - r[0][0], r[1][1] - r[0][1], r[1][2] - r[0][2]};
        const double e2[3] = {r[2][0] - r[0][0], r[2][1] - r[0][1], r[2][2] - r[0][2]};
        const double cx = e1[1] * e2[2] - e1[2] * e2[1], cy = e1[2] * e2[0] - e1[0] * e2[2],
                     cz = e1[0] * e2[1] - e1[1] * e2[0];
        const double A = 0.5 * std::sqrt(cx * cx + cy * cy + cz * cz);
        asoft[t] = selfAlpha * std::sqrt(A / kPi);
    }
    std::vector<Side> side(2 * (size_t)Ne);
    for (int e = 0; e < Ne; e++) {
        for (int sd = 0; sd < 2; sd++) {
            Side &o = side[2 * (size_t)e + sd];
            std::memset(&o, 0, sizeof(Side));
            const int t = sd == 0 ? mesh->plusTri[e] : mesh->minusTri[e];
            const double A = sd == 0 ? mesh->Ap[e] : mesh->Am[e];
            o.t = t;
            o.w = t > 0 ? A : 0.0;
            if (t > 0) {
                o.px = cent[3 * (t - 1)];
                o.py = cent[3 * (t - 1) + 1];
                o.pz = cent[3 * (t - 1) + 2];
            }
            if (t > 0 && A > 0) {
                const double l = mesh->len[e];
                const int sg = sd == 0 ? mesh->plusSign[e] : mesh->minusSign[e];
                const double sc = (double)sg * (l / (2.0 * A));
                const double *v = sd == 0 ? mesh->rp : mesh->rm;
                const double vx = v[e], vy = v[e + Ne], vz = v[e + 2 * (size_t)Ne];
                if (sd == 0) {
                    o.fx = sc * (o.px - vx); o.fy = sc * (o.py - vy); o.fz = sc * (o.pz - vz);
                    o.div = (double)sg * (l / A);
                } else {
                    o.fx = sc * (vx - o.px); o.fy = sc * (vy - o.py); o.fz = sc * (vz - o.pz);
                    o.div = (double)sg * (-(l / A));
                }
            }
        }
    }
    const size_t side_bytes = sizeof(Side) * side.size();
    EFIE_TRY(scratch.reserve(side_bytes + sizeof(double) * Nt + 256));
    char *base = scratch.as<char>();
    EFIE_CUDA(cudaMemcpyAsync(base, side.data(), side_bytes, cudaMemcpyHostToDevice, ctx->stream));
    double *d_asoft = reinterpret_cast<double *>(base + ((side_bytes + 255) / 256) * 256);
    EFIE_CUDA(cudaMemcpyAsync(d_asoft, asoft.data(), sizeof(double) * Nt, cudaMemcpyHostToDevice, ctx->stream));
    dim3 gg((Ne + 63) / 64, (Ne + 3) / 4);
    size_t tok = ctx->log.begin(ctx->stream);
    k_centroid_z<<<gg, 256, 0, ctx->stream>>>(Ne, reinterpret_cast<const Side *>(base), d_asoft, ph.kr, ph.ki, ph.alr,
                                              ph.ali, ph.ber, ph.bei, static_cast<double2 *>(Z));
    EFIE_CUDA(cudaGetLastError());
    ctx->log.end(EFIE_K_QUAD, ctx->stream, tok, 4.0 * (double)Ne * Ne);
    return EFIE_OK;
}
