// Mixed-precision dense solve of Z x = V on sm_100a, batched over frequencies.
//
// The reference factors Z in complex128 with cusolverDnZgetrf/Zgetrs
// (patch_sweep_fastquad_cuda.cu:765-771), one frequency at a time.  Here a
// batch of B frequencies is solved together: Z_f (complex128, column-major,
// as assembled) is kept for the residual, and a complex64 copy of each Z_f is
// factored without pivoting (Z is complex symmetric and, for these EFIE
// matrices, strongly diagonal: element growth stays near 1); FP64 iterative
// refinement then recovers the complex128 solution:
//     x = 0, r = V;  repeat { d = U^-1 L^-1 r (complex64);  x += d;
//                            r = V - Z x (complex128) }  until ||r|| <= tol ||V||.
// Every kernel carries the frequency in its grid (blockIdx.z or blockIdx.x),
// so the latency-bound parts of B problems (diagonal blocks, triangular-solve
// chains, small trailing updates) overlap instead of serialising.  A zero
// pivot or a refinement that stalls makes the caller re-solve that frequency
// with the complex128 LU.
//
// Working matrix of frequency f: two FP32 planes (re, im), row-major,
// leading dimension ld (multiple of 64), at planes + f * pstride.
#include <algorithm>
#include <cmath>
#include <vector>

#include <cuda_fp16.h>

#include "efie_internal.h"
#include "solve.h"

namespace {

constexpr int NB = 64;   // diagonal block size of the LU and the triangular solves
constexpr size_t kTwoTiles = sizeof(float2) * 2 * NB * (NB + 1);
// k_panels' tiles: rows padded to 66 complex (528 bytes, a multiple of 16) so
// that two consecutive entries of a row load as one float4
constexpr int PS = NB + 2;
constexpr size_t kPanelSmem = sizeof(float2) * 2 * NB * PS;

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// ---------------------------------------------------------------------------
// Z_f (c128, column-major) -> planes_f (row-major).  32x32 tiles, grid z = f.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_z_to_planes(int N, const double2 *__restrict__ Z, size_t zstride,
                                                     float *__restrict__ planes, size_t pstride, int ld) {
    __shared__ float tr[32][33], ti[32][33];
    const int f = blockIdx.z;
    Z += zstride * f;
    float *Ar = planes + pstride * f, *Ai = Ar + (size_t)ld * N;
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;  // bx: column block, by: row block
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int r = ty; r < 32; r += 8) {
        const int row = by + tx, col = bx + r;  // coalesced along the columns of Z
        double2 v = (row < N && col < N) ? Z[(size_t)row + (size_t)N * col] : make_double2(0, 0);
        tr[r][tx] = (float)v.x;
        ti[r][tx] = (float)v.y;
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const int row = by + r, col = bx + tx;  // coalesced along the rows of the planes
        if (row < N && col < N) {
            Ar[(size_t)row * ld + col] = tr[tx][r];
            Ai[(size_t)row * ld + col] = ti[tx][r];
        }
    }
}

// ---------------------------------------------------------------------------
// Diagonal block bi of every frequency (blockIdx.x = f): LU without pivoting
// of A[k:k+kb, k:k+kb] (identity beyond kb) and the inverses of its unit-lower
// L and upper U factors (kept for the panel products and the triangular
// solves), blocked by 16 in shared memory.  For each 16-column panel one warp
// factors it in registers (lane l holds rows o + l and o + 32 + l; the pivot
// row is broadcast by shuffles, so its 16 steps need no barrier), then the
// 16-row U strip (forward substitution, one thread per column) and the
// trailing block (one rank-16 update) follow, one barrier each.  The inverses
// are built the same way: the four 16 x 16 diagonal blocks of L^-1 and U^-1
// by substitution (one warp per block, one lane per column), then the
// off-diagonal blocks block row by block row,
//     X_ij = -X_ii sum_{j<=m<i} L_im X_mj     (L^-1, i > j, downwards)
//     Y_ij = -Y_ii sum_{i<m<=j} U_im Y_mj     (U^-1, i < j, upwards),
// block row r of L^-1 with block row 3 - r of U^-1: 20 barriers in all.
// ---------------------------------------------------------------------------
constexpr int SB = 16;   // sub-block of the diagonal factorisation
constexpr size_t kDiagSmem = sizeof(float2) * (3 * NB * (NB + 1) + 2 * 3 * SB * (SB + 1));

__device__ __forceinline__ void cfms(float2 &acc, float2 l, float2 u) {   // acc -= l * u
    acc.x -= l.x * u.x - l.y * u.y;
    acc.y -= l.x * u.y + l.y * u.x;
}

__device__ __forceinline__ void cfma(float2 &acc, float2 l, float2 u) {   // acc += l * u
    acc.x += l.x * u.x - l.y * u.y;
    acc.y += l.x * u.y + l.y * u.x;
}

__device__ __forceinline__ float2 shfl2(float2 v, int src) {
    return make_float2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

// 1 / p for complex p; `zero` when |p|^2 is not positive
__device__ __forceinline__ float2 crecip(float2 p, bool &zero) {
    const float den = p.x * p.x + p.y * p.y;
    zero = !(den > 0.f);
    const float rd = 1.0f / den;
    return make_float2(p.x * rd, -p.y * rd);
}

__global__ void __launch_bounds__(256) k_diag_factor(int N, int k, int kb, int bi, float *__restrict__ planes,
                                                     size_t pstride, int ld, float2 *__restrict__ dinv,
                                                     size_t dstride, char *__restrict__ ctl,
                                                     const int *__restrict__ active, int sym) {
    const int f = blockIdx.x;
    if (!active[f]) return;
    extern __shared__ float2 dsm[];
    float2(*A)[NB + 1] = reinterpret_cast<float2(*)[NB + 1]>(dsm);   // the block, then L\U
    float2(*X)[NB + 1] = A + NB;                                        // L^-1
    float2(*Y)[NB + 1] = A + 2 * NB;                                    // U^-1
    float2(*TX)[SB][SB + 1] = reinterpret_cast<float2(*)[SB][SB + 1]>(dsm + 3 * NB * (NB + 1));
    float2(*TY)[SB][SB + 1] = TX + 3;   // partial sums of the off-diagonal inverse blocks
    float *Ar = planes + pstride * f, *Ai = Ar + (size_t)ld * N;
    float2 *Linv = dinv + dstride * f + (size_t)bi * 2 * NB * NB, *Uinv = Linv + NB * NB;
    int *err = reinterpret_cast<int *>(ctl + 64 * f + 36);
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;

    for (int e = t; e < NB * NB; e += 256) {
        const int r = e >> 6, c = e & 63;
        float2 v = make_float2(r == c ? 1.f : 0.f, 0.f);   // identity beyond kb
        if (r < kb && c < kb) {
            // symmetric Z: the lower triangle, mirrored
            const int rr = (sym && c > r) ? c : r, cc = (sym && c > r) ? r : c;
            const size_t o = (size_t)(k + rr) * ld + k + cc;
            v = make_float2(Ar[o], Ai[o]);
        }
        A[r][c] = v;
        X[r][c] = make_float2(0.f, 0.f);
        Y[r][c] = make_float2(0.f, 0.f);
    }
    __syncthreads();

    // ---- LU without pivoting ----
    bool bad = false;
    for (int p = 0; p < NB / SB; p++) {
        const int o = p * SB;
        if (warp == 0) {
            const int i0 = o + lane, i1 = o + 32 + lane;
            const bool h0 = i0 < NB, h1 = i1 < NB;
            float2 a0[SB], a1[SB];
#pragma unroll
            for (int c = 0; c < SB; c++) {
                a0[c] = h0 ? A[i0][o + c] : make_float2(0.f, 0.f);
                a1[c] = h1 ? A[i1][o + c] : make_float2(0.f, 0.f);
            }
#pragma unroll
            for (int j = 0; j < SB; j++) {
                float2 u[SB];
                // row o + j sits in lane j; symmetric Z (L D L^T): the row is
                // the column below the pivot, row o + c in lane c
                u[j] = shfl2(a0[j], j);
#pragma unroll
                for (int c = j + 1; c < SB; c++) u[c] = sym == 1 ? shfl2(a0[j], c) : shfl2(a0[c], j);
                bool z;
                const float2 inv = crecip(u[j], z);
                bad |= z;
                if (sym == 1 && lane == j) {
#pragma unroll
                    for (int c = j + 1; c < SB; c++) a0[c] = u[c];
                }
                if (lane > j) {
                    const float2 l = cmulf(a0[j], inv);
                    a0[j] = l;
#pragma unroll
                    for (int c = j + 1; c < SB; c++) cfms(a0[c], l, u[c]);
                }
                const float2 l = cmulf(a1[j], inv);
                a1[j] = l;
#pragma unroll
                for (int c = j + 1; c < SB; c++) cfms(a1[c], l, u[c]);
            }
#pragma unroll
            for (int c = 0; c < SB; c++) {
                if (h0) A[i0][o + c] = a0[c];
                if (h1) A[i1][o + c] = a1[c];
            }
        }
        __syncthreads();
        const int w = NB - o - SB;   // columns (rows) right of (below) the panel
        if (sym == 1 && t < w) {     // U strip of L D L^T: U[o + i][c] = d_i L[c][o + i]
            const int c = o + SB + t;
#pragma unroll
            for (int i = 0; i < SB; i++) A[o + i][c] = cmulf(A[o + i][o + i], A[c][o + i]);
        } else if (t < w) {          // U strip: forward substitution with the panel's unit-lower block
            const int c = o + SB + t;
            float2 x[SB];
#pragma unroll
            for (int i = 0; i < SB; i++) {
                float2 v = A[o + i][c];
#pragma unroll
                for (int m = 0; m < i; m++) cfms(v, A[o + i][o + m], x[m]);
                x[i] = v;
                A[o + i][c] = v;
            }
        }
        __syncthreads();
        for (int e = t; e < w * w; e += 256) {   // trailing block: rank-16 update
            const int i = o + SB + e / w, c = o + SB + e % w;
            float2 v = A[i][c];
#pragma unroll
            for (int m = 0; m < SB; m++) cfms(v, A[i][o + m], A[o + m][c]);
            A[i][c] = v;
        }
        __syncthreads();
    }

    // ---- inverses: diagonal 16 x 16 blocks ----
    if (lane < SB) {
        const int c = lane;
        if (warp < 4) {   // L^-1: unit lower, forward substitution
            const int o = warp * SB;
            float2 x[SB];
#pragma unroll
            for (int i = 0; i < SB; i++) {
                float2 v = make_float2(i == c ? 1.f : 0.f, 0.f);
#pragma unroll
                for (int m = 0; m < i; m++) cfms(v, A[o + i][o + m], x[m]);
                x[i] = v;
                X[o + i][o + c] = v;
            }
        } else {          // U^-1: upper, backward substitution
            const int o = (warp - 4) * SB;
            float2 y[SB];
#pragma unroll
            for (int i = SB - 1; i >= 0; i--) {
                float2 v = make_float2(i == c ? 1.f : 0.f, 0.f);
#pragma unroll
                for (int m = i + 1; m < SB; m++) cfms(v, A[o + i][o + m], y[m]);
                bool z;
                v = cmulf(v, crecip(A[o + i][o + i], z));
                y[i] = v;
                Y[o + i][o + c] = v;
            }
        }
    }
    __syncthreads();
    // ---- inverses: off-diagonal blocks, L^-1 row R = r with U^-1 row Q = 3 - r ----
    for (int r = 1; r < NB / SB; r++) {
        const int R = r, Q = NB / SB - 1 - r, nx = r * SB * SB;
        for (int e = t; e < 2 * nx; e += 256) {
            const bool isx = e < nx;
            const int e2 = isx ? e : e - nx;
            const int jb = e2 >> 8, a = (e2 >> 4) & 15, b = e2 & 15;
            float2 v = make_float2(0.f, 0.f);
            if (isx) {   // -sum_{jb<=m<R} L_Rm X_m,jb
                for (int m = jb; m < R; m++)
#pragma unroll
                    for (int q = 0; q < SB; q++) cfms(v, A[R * SB + a][m * SB + q], X[m * SB + q][jb * SB + b]);
                TX[jb][a][b] = v;
            } else {     // -sum_{Q<m<=j} U_Qm Y_mj, j = Q + 1 + jb
                const int j = Q + 1 + jb;
                for (int m = Q + 1; m <= j; m++)
#pragma unroll
                    for (int q = 0; q < SB; q++) cfms(v, A[Q * SB + a][m * SB + q], Y[m * SB + q][j * SB + b]);
                TY[jb][a][b] = v;
            }
        }
        __syncthreads();
        for (int e = t; e < 2 * nx; e += 256) {
            const bool isx = e < nx;
            const int e2 = isx ? e : e - nx;
            const int jb = e2 >> 8, a = (e2 >> 4) & 15, b = e2 & 15;
            float2 v = make_float2(0.f, 0.f);
            if (isx) {
#pragma unroll
                for (int q = 0; q < SB; q++) cfma(v, X[R * SB + a][R * SB + q], TX[jb][q][b]);
                X[R * SB + a][jb * SB + b] = v;
            } else {
#pragma unroll
                for (int q = 0; q < SB; q++) cfma(v, Y[Q * SB + a][Q * SB + q], TY[jb][q][b]);
                Y[Q * SB + a][(Q + 1 + jb) * SB + b] = v;
            }
        }
        __syncthreads();
    }

    if (sym == 1) {
        // U = D L^T: U^-1 = L^-T D^-1 from L^-1, so that U^-1 L^-1 is
        // symmetric as the inverse of a symmetric block is
        for (int e = t; e < NB * NB; e += 256) {
            const int r = e >> 6, c = e & 63;
            bool z;
            Y[r][c] = r <= c ? cmulf(X[c][r], crecip(A[c][c], z)) : make_float2(0.f, 0.f);
        }
        __syncthreads();
    }
    // ---- factors back to the planes, inverses to their slots ----
    for (int e = t; e < NB * NB; e += 256) {
        const int r = e >> 6, c = e & 63;
        if (r < kb && c < kb) {
            const size_t o = (size_t)(k + r) * ld + k + c;
            Ar[o] = A[r][c].x;
            Ai[o] = A[r][c].y;
        }
        Linv[e] = X[r][c];
        Uinv[e] = Y[r][c];
    }
    if (t == 0 && bad) atomicExch(err, 1);
}

// A finished 64 x 64 factor block (thread (ty, tx) holds rows ty + 16 a,
// columns tx + 16 b) as tensor-core operand of the panel chain's updates
// (K = 64): rows of L (columns of U when ublk) scaled by the power of two of
// their maximum mx, split into FP16 hi + lo, in the packed layout
// [chunk][re hi, re lo, im hi, im lo][row][32] with the 64-byte swizzle,
// staged in `pk` (32 KB of shared memory), then the eight 64-row component
// blocks (4 KB each) to their planes at `dst`.
__device__ __forceinline__ void emit_block(const float2 (&acc)[4][4], bool ublk, const float *mx, __half *pk,
                                           __half *dst, int ippitch, int tid, int ty, int tx) {
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) {
            const int i = ty + 16 * a, j = tx + 16 * b;
            const int prow = ublk ? j : i, kidx = ublk ? i : j;
            const float sc = efie_pow2_scale(mx[prow]);
            const int chunk = kidx >> 5, kq = kidx & 31;
            const int o = chunk * 4 * NB * 32 + (int)(efie_swz64(prow, kq) >> 1);
            __half h, l;
            const float vr = acc[a][b].x * sc, vi = acc[a][b].y * sc;
            h = __float2half_rn(vr);
            l = __float2half_rn(vr - __half2float(h));
            pk[o] = h;
            pk[o + NB * 32] = l;
            h = __float2half_rn(vi);
            l = __float2half_rn(vi - __half2float(h));
            pk[o + 2 * NB * 32] = h;
            pk[o + 3 * NB * 32] = l;
        }
    __syncthreads();
    for (int e = tid; e < 8 * NB * 32 / 8; e += 256) {
        const int blk = e / (NB * 32 / 8), q = e % (NB * 32 / 8);
        reinterpret_cast<float4 *>(dst + (size_t)blk * ippitch * 32)[q] =
            reinterpret_cast<const float4 *>(pk + blk * NB * 32)[q];
    }
}

// ---------------------------------------------------------------------------
// Panels: U12 = Linv * A12 (row panel) and L21 = A21 * Uinv (column panel).
// One 64x64 tile per CTA, in place.  blockIdx.y: 0 row panel, 1 column panel;
// blockIdx.z: frequency.  Symmetric Z (sym): one CTA per tile of the column
// panel forms U12 = Linv * A21^T and from it L21 = U12^T D^-1.  Thread
// (ty, tx) = (t / 16, t mod 16) computes rows
// ty + 16a and columns tx + 16b (a, b < 4): the 16 threads of a half-warp
// read 16 consecutive complex entries of a shared-memory row, which is
// conflict-free for 64-bit loads.  Tiles are loaded with float4 reads of
// the re/im planes (rows are 16-byte aligned: ld and the offsets are
// multiples of 64).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256, 3) k_panels(int N, int k, int kb, int bi, float *__restrict__ planes,
                                                size_t pstride, int ld, const float2 *__restrict__ dinv,
                                                size_t dstride, const int *__restrict__ active,
                                                float *__restrict__ lmax, float *__restrict__ umax,
                                                size_t mstride, int nblk, __half *__restrict__ ipl,
                                                __half *__restrict__ ipu, size_t ipstride, int ippitch,
                                                int emit, int sym, int kend) {
    const int f = blockIdx.z;
    if (!active[f]) return;
    extern __shared__ float2 dyn[];
    float2(*M)[PS] = reinterpret_cast<float2(*)[PS]>(dyn);             // the inverse
    float2(*T)[PS] = reinterpret_cast<float2(*)[PS]>(dyn + NB * PS);  // the panel tile
    float *Ar = planes + pstride * f, *Ai = Ar + (size_t)ld * N;
    const float2 *Linv = dinv + dstride * f + (size_t)bi * 2 * NB * NB, *Uinv = Linv + NB * NB;
    const int tid = threadIdx.x;
    const bool rowp = !sym && blockIdx.y == 0;
    const int off = k + kb + blockIdx.x * NB;
    if (off >= N) return;
    const int ext = min(NB, N - off);
    auto load_inverse = [&](const float2 *src) {
        const float4 *inv4 = reinterpret_cast<const float4 *>(src);   // 2 complex per float4
        for (int e = tid; e < NB * NB / 2; e += 256) {
            const float4 v = inv4[e];
            const int i = (2 * e) / NB, j = (2 * e) % NB;
            M[i][j] = make_float2(v.x, v.y);
            M[i][j + 1] = make_float2(v.z, v.w);
        }
    };
    load_inverse((rowp || sym) ? Linv : Uinv);
    // tile rows: row panel rows k..k+kb (columns off..off+ext); column panel rows off..off+ext (columns k..k+kb)
    const int nrow = rowp ? kb : ext, ncol = rowp ? ext : kb;
    const size_t base = rowp ? (size_t)k * ld + off : (size_t)off * ld + k;
    for (int e = tid; e < NB * NB / 4; e += 256) {
        const int i = e >> 4, j = (e & 15) * 4;
        float4 re = make_float4(0.f, 0.f, 0.f, 0.f), im = re;
        if (i < nrow && j < ncol) {
            re = *reinterpret_cast<const float4 *>(Ar + base + (size_t)i * ld + j);
            im = *reinterpret_cast<const float4 *>(Ai + base + (size_t)i * ld + j);
        }
        T[i][j] = make_float2(re.x, im.x);
        T[i][j + 1] = make_float2(re.y, im.y);
        T[i][j + 2] = make_float2(re.z, im.z);
        T[i][j + 3] = make_float2(re.w, im.w);
    }
    __syncthreads();
    const int ty = tid >> 4, tx = tid & 15;
    if (sym) {
        // U[k + i][off + j] = sum_q Linv[i][q] T[j][q] (T: rows off.. of the
        // lower part), and with U^-1 = L^-T D^-1 the column panel follows
        // from it exactly: L[off + j][k + i] = U[i][j] / d_i.  Only U is kept
        // in registers; L is formed from it where it is used, so the kernel
        // fits three CTAs per SM.
        __shared__ float umx[NB], lmx[NB];
        __shared__ float2 rdiag[NB];
        if (tid < NB) rdiag[tid] = Uinv[tid * NB + tid];   // 1 / d_i
        float2 au[4][4];
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
            for (int b = 0; b < 4; b++) au[a][b] = make_float2(0.f, 0.f);
        // two steps of q per pass: entries q, q + 1 of a row are one float4
#pragma unroll 2
        for (int q = 0; q < NB; q += 2) {
            float4 x[4], y[4];
#pragma unroll
            for (int a = 0; a < 4; a++) {
                x[a] = *reinterpret_cast<const float4 *>(&M[ty + 16 * a][q]);
                y[a] = *reinterpret_cast<const float4 *>(&T[tx + 16 * a][q]);
            }
#pragma unroll
            for (int a = 0; a < 4; a++)
#pragma unroll
                for (int b = 0; b < 4; b++) {
                    cfma(au[a][b], make_float2(x[a].x, x[a].y), make_float2(y[b].x, y[b].y));
                    cfma(au[a][b], make_float2(x[a].z, x[a].w), make_float2(y[b].z, y[b].w));
                }
        }
        __syncthreads();   // M, T and rdiag: M and T are free from here
        // the maxima's partial reductions live in M until the L rows are out
        float(*ured)[17] = reinterpret_cast<float(*)[17]>(&M[0][0]);
        float(*lred)[17] = ured + NB;
        float cu[4] = {0.f, 0.f, 0.f, 0.f}, cl[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
            for (int b = 0; b < 4; b++) {
                const int i = ty + 16 * a, j = tx + 16 * b;
                const float2 l = cmulf(au[a][b], rdiag[i]);
                T[j][i] = l;   // L tile, row j
                if (i < kb && j < ext) {
                    const size_t o = (size_t)(k + i) * ld + off + j;
                    Ar[o] = au[a][b].x;
                    Ai[o] = au[a][b].y;
                    cu[b] = fmaxf(cu[b], fmaxf(fabsf(au[a][b].x), fabsf(au[a][b].y)));
                    cl[b] = fmaxf(cl[b], fmaxf(fabsf(l.x), fabsf(l.y)));
                }
            }
#pragma unroll
        for (int b = 0; b < 4; b++) {
            ured[tx + 16 * b][ty] = cu[b];
            lred[tx + 16 * b][ty] = cl[b];
        }
        __syncthreads();
        // L rows off.. (columns k..k+kb): consecutive threads, consecutive columns
        for (int e = tid; e < NB * NB; e += 256) {
            const int r = e >> 6, c = e & (NB - 1);
            if (r < ext && c < kb) {
                const size_t o = (size_t)(off + r) * ld + k + c;
                Ar[o] = T[r][c].x;
                Ai[o] = T[r][c].y;
            }
        }
        if (tid < NB) {
            float mu = 0.f, ml = 0.f;
#pragma unroll
            for (int q = 0; q < 16; q++) mu = fmaxf(mu, ured[tid][q]), ml = fmaxf(ml, lred[tid][q]);
            umx[tid] = mu;
            lmx[tid] = ml;
            if (tid < ext) {
                umax[mstride * f + (size_t)bi * ld + off + tid] = mu;
                lmax[mstride * f + (size_t)(off + tid) * nblk + bi] = ml;
            }
        }
        __syncthreads();   // T (the L staging) and M (the partial maxima) are free
        if (!emit) return;
        // operands of the panel chain's update: the U block when its columns
        // lie inside the panel, then the L rows (columns of the U tile) always
        if (off < kend)
            emit_block(au, true, umx, reinterpret_cast<__half *>(&M[0][0]),
                       ipu + ipstride * f + (size_t)(off - k - kb) * 32, ippitch, tid, ty, tx);
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
            for (int b = 0; b < 4; b++) au[a][b] = cmulf(au[a][b], rdiag[ty + 16 * a]);
        emit_block(au, true, lmx, reinterpret_cast<__half *>(&T[0][0]),
                   ipl + ipstride * f + (size_t)(off - k - kb) * 32, ippitch, tid, ty, tx);
        return;
    }
    float2 acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) acc[a][b] = make_float2(0.f, 0.f);
    // row panel: out = M * T; column panel: out = T * M
    const float2(*X)[PS] = rowp ? M : T;
    const float2(*Y)[PS] = rowp ? T : M;
#pragma unroll 4
    for (int q = 0; q < NB; q++) {
        float2 x[4], y[4];
#pragma unroll
        for (int a = 0; a < 4; a++) {
            x[a] = X[ty + 16 * a][q];
            y[a] = Y[q][tx + 16 * a];
        }
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
            for (int b = 0; b < 4; b++) {
                acc[a][b].x += x[a].x * y[b].x - x[a].y * y[b].y;
                acc[a][b].y += x[a].x * y[b].y + x[a].y * y[b].x;
            }
    }
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) {
            const int i = ty + 16 * a, j = tx + 16 * b;
            if (i < nrow && j < ncol) {
                Ar[base + (size_t)i * ld + j] = acc[a][b].x;
                Ai[base + (size_t)i * ld + j] = acc[a][b].y;
            }
        }
    // maxima of the finished factor block: per column of the U block (row panel)
    // or per row of the L block (column panel), over its 64 rows / columns
    __shared__ float red[NB][17];
    __shared__ float mx[NB];
    __syncthreads();   // M and T are no longer read
    float mag[4][4];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) {
            const int i = ty + 16 * a, j = tx + 16 * b;
            mag[a][b] = (i < nrow && j < ncol) ? fmaxf(fabsf(acc[a][b].x), fabsf(acc[a][b].y)) : 0.f;
        }
    if (rowp) {
#pragma unroll
        for (int b = 0; b < 4; b++)
            red[tx + 16 * b][ty] = fmaxf(fmaxf(mag[0][b], mag[1][b]), fmaxf(mag[2][b], mag[3][b]));
    } else {
#pragma unroll
        for (int a = 0; a < 4; a++)
            red[ty + 16 * a][tx] = fmaxf(fmaxf(mag[a][0], mag[a][1]), fmaxf(mag[a][2], mag[a][3]));
    }
    __syncthreads();
    if (tid < NB) {
        float m = 0.f;
#pragma unroll
        for (int q = 0; q < 16; q++) m = fmaxf(m, red[tid][q]);
        mx[tid] = m;
        if (rowp) {
            if (tid < ncol) umax[mstride * f + (size_t)bi * ld + off + tid] = m;
        } else {
            if (tid < nrow) lmax[mstride * f + (size_t)(off + tid) * nblk + bi] = m;
        }
    }
    if (!emit) return;
    __syncthreads();   // T is no longer read: the staging of the pack
    emit_block(acc, rowp, mx, reinterpret_cast<__half *>(&T[0][0]),
               (rowp ? ipu : ipl) + ipstride * f + (size_t)(off - k - kb) * 32, ippitch, tid, ty, tx);
}

// ---------------------------------------------------------------------------
// C[r0:r1, c0:c1] -= L[r0:r1, kcol:kcol+K] * U[krow:krow+K, c0:c1] on CUDA
// cores (complex FP32), 64x64 tiles, K <= 64: small blocks and the portable path.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_update_simt(int N, int r0, int r1, int c0, int c1, int kcol, int krow, int K,
                                                     float *__restrict__ planes, size_t pstride, int ld,
                                                     const int *__restrict__ active) {
    const int f = blockIdx.z;
    if (!active[f]) return;
    extern __shared__ float2 dyn[];
    float2(*Ls)[NB + 1] = reinterpret_cast<float2(*)[NB + 1]>(dyn);
    float2(*Us)[NB + 1] = reinterpret_cast<float2(*)[NB + 1]>(dyn + NB * (NB + 1));
    float *Ar = planes + pstride * f, *Ai = Ar + (size_t)ld * N;
    const int tid = threadIdx.x;
    const int row0 = r0 + blockIdx.y * NB, col0 = c0 + blockIdx.x * NB;
    if (row0 >= r1 || col0 >= c1) return;
    for (int e = tid; e < NB * NB; e += 256) {
        const int i = e / NB, j = e % NB;
        Ls[i][j] = (row0 + i < r1 && j < K)
                       ? make_float2(Ar[(size_t)(row0 + i) * ld + kcol + j], Ai[(size_t)(row0 + i) * ld + kcol + j])
                       : make_float2(0.f, 0.f);
        Us[i][j] = (i < K && col0 + j < c1)
                       ? make_float2(Ar[(size_t)(krow + i) * ld + col0 + j], Ai[(size_t)(krow + i) * ld + col0 + j])
                       : make_float2(0.f, 0.f);
    }
    __syncthreads();
    const int rr = (tid >> 4) * 4, cc = (tid & 15) * 4;
    float2 acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) acc[a][b] = make_float2(0.f, 0.f);
    for (int q = 0; q < K; q++) {
        float2 x[4], y[4];
#pragma unroll
        for (int a = 0; a < 4; a++) {
            x[a] = Ls[rr + a][q];
            y[a] = Us[q][cc + a];
        }
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
            for (int b = 0; b < 4; b++) {
                acc[a][b].x += x[a].x * y[b].x - x[a].y * y[b].y;
                acc[a][b].y += x[a].x * y[b].y + x[a].y * y[b].x;
            }
    }
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) {
            const int i = row0 + rr + a, j = col0 + cc + b;
            if (i < r1 && j < c1) {
                Ar[(size_t)i * ld + j] -= acc[a][b].x;
                Ai[(size_t)i * ld + j] -= acc[a][b].y;
            }
        }
}

// ---------------------------------------------------------------------------
// r_f = V - Z_f x_f (complex128 GEMV over the column-major Z_f), the complex64
// copy of r_f for the next correction, and ||r_f||.  Block = 32 rows x 8
// column groups, grid y = f.  The last CTA of frequency f turns ||r_f|| into
// its convergence flag (ctl_f: red[3] @0, counter @24, conv @28, skip @32).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_residual(int N, const double2 *__restrict__ Zb, size_t zstride,
                                                  const double2 *__restrict__ xb, const double2 *__restrict__ b,
                                                  float2 *__restrict__ rfb, int vstride, char *__restrict__ ctl,
                                                  double tol, double2 *__restrict__ routb,
                                                  double *__restrict__ partb) {
    const int f = blockIdx.y;
    char *c = ctl + 64 * f;
    double *red = reinterpret_cast<double *>(c);
    unsigned int *counter = reinterpret_cast<unsigned int *>(c + 24);
    int *conv = reinterpret_cast<int *>(c + 28);
    int *skip = reinterpret_cast<int *>(c + 32);
    if (*skip) return;
    const double2 *Z = Zb + zstride * f;
    const double2 *x = xb + (size_t)N * f;
    float2 *rf = rfb + (size_t)vstride * f;
    __shared__ double2 part[8][32];
    __shared__ double sq[32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, g = threadIdx.x >> 5;
    const int m = blockIdx.x * 32 + lane;
    double2 s = make_double2(0.0, 0.0);
    if (m < N) {
        for (int n = g; n < N; n += 8) {
            const double2 z = Z[(size_t)m + (size_t)N * n];
            const double2 v = x[n];
            s.x += z.x * v.x - z.y * v.y;
            s.y += z.x * v.y + z.y * v.x;
        }
    }
    part[g][lane] = s;
    __syncthreads();
    if (g == 0) {
        double2 t = make_double2(0.0, 0.0);
        for (int i = 0; i < 8; i++) {
            t.x += part[i][lane].x;
            t.y += part[i][lane].y;
        }
        double q = 0.0;
        if (m < N) {
            const double2 bb = b[m];
            const double2 r = make_double2(bb.x - t.x, bb.y - t.y);
            rf[m] = make_float2((float)r.x, (float)r.y);
            if (routb) routb[(size_t)N * f + m] = r;
            q = r.x * r.x + r.y * r.y;
        }
        sq[lane] = q;
    }
    __syncthreads();
    // per-CTA partial sums, added in CTA order by the last CTA: the norm (and
    // with it every later rounding) does not depend on the CTA schedule
    double *part_f = partb + (size_t)gridDim.x * f;
    if (threadIdx.x == 0) {
        double q = 0.0;
        for (int i = 0; i < 32; i++) q += sq[i];
        part_f[blockIdx.x] = q;
        __threadfence();
        const unsigned int done = atomicAdd(counter, 1u);
        last = (done == gridDim.x - 1);
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        double acc = 0.0;
        for (unsigned int i = 0; i < gridDim.x; i++) acc += ((volatile double *)part_f)[i];
        const double rr = sqrt(acc);
        const double rel = rr / red[1];
        red[2] = rel;
        red[0] = 0.0;
        *counter = 0u;
        if (rel <= tol) {
            *conv = 1;
            *skip = 1;
        }
    }
}

// r_f = b - y_f for a precomputed y_f = Z_f x_f; the rest as k_residual
// (complex64 copy, optional complex128 copy, ||r_f|| summed in CTA order by
// the last CTA, convergence flags).  Block = 256 rows, grid (rows / 256, B).
__global__ void __launch_bounds__(256) k_resid_finish(int N, const double2 *__restrict__ yb,
                                                      const double2 *__restrict__ b, float2 *__restrict__ rfb,
                                                      int vstride, char *__restrict__ ctl, double tol,
                                                      double2 *__restrict__ routb, double *__restrict__ partb) {
    const int f = blockIdx.y;
    char *c = ctl + 64 * f;
    double *red = reinterpret_cast<double *>(c);
    unsigned int *counter = reinterpret_cast<unsigned int *>(c + 24);
    int *conv = reinterpret_cast<int *>(c + 28);
    int *skip = reinterpret_cast<int *>(c + 32);
    if (*skip) return;
    __shared__ double sq[8];
    __shared__ bool last;
    const int m = blockIdx.x * 256 + threadIdx.x;
    double q = 0.0;
    if (m < N) {
        const double2 y = yb[(size_t)N * f + m], bb = b[m];
        const double2 r = make_double2(bb.x - y.x, bb.y - y.y);
        rfb[(size_t)vstride * f + m] = make_float2((float)r.x, (float)r.y);
        if (routb) routb[(size_t)N * f + m] = r;
        q = r.x * r.x + r.y * r.y;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) q += __shfl_xor_sync(0xffffffffu, q, o);
    if ((threadIdx.x & 31) == 0) sq[threadIdx.x >> 5] = q;
    __syncthreads();
    double *part_f = partb + (size_t)gridDim.x * f;
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < 8; i++) t += sq[i];
        part_f[blockIdx.x] = t;
        __threadfence();
        const unsigned int done = atomicAdd(counter, 1u);
        last = (done == gridDim.x - 1);
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        double acc = 0.0;
        for (unsigned int i = 0; i < gridDim.x; i++) acc += ((volatile double *)part_f)[i];
        const double rel = sqrt(acc) / red[1];
        red[2] = rel;
        red[0] = 0.0;
        *counter = 0u;
        if (rel <= tol) {
            *conv = 1;
            *skip = 1;
        }
    }
}

// ---------------------------------------------------------------------------
// Port reduction + Zin/S11 (patch_sweep_fastquad_cuda.cu:777-799 for the
// Gaussian model; patch_sweep_cuda.cu:484-494 for the edge difference).
// One CTA per frequency.  out_f = {Zin, S11}.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_port(int N, const double2 *__restrict__ xb, const double *__restrict__ wport,
                                               int model, int pe, int ge, double V0, double Z0,
                                               double2 *__restrict__ out) {
    __shared__ double sr[1024], si[1024];
    const int f = blockIdx.x;
    const double2 *x = xb + (size_t)N * f;
    const int tid = threadIdx.x;
    double a = 0.0, c = 0.0;
    if (model == EFIE_PORT_GAUSS) {
        for (int i = tid; i < N; i += 1024) {
            a += wport[i] * x[i].x;
            c += wport[i] * x[i].y;
        }
    }
    sr[tid] = a;
    si[tid] = c;
    __syncthreads();
    for (int o = 512; o > 0; o >>= 1) {
        if (tid < o) {
            sr[tid] += sr[tid + o];
            si[tid] += si[tid + o];
        }
        __syncthreads();
    }
    if (tid == 0) {
        double Ipr = sr[0], Ipi = si[0];
        if (model == EFIE_PORT_EDGE_DIFF) {
            Ipr = x[pe].x - x[ge].x;
            Ipi = x[pe].y - x[ge].y;
        }
        const double den = Ipr * Ipr + Ipi * Ipi;
        const double Zr = V0 * (Ipr / den), Zi = -V0 * (Ipi / den);
        const double ar = Zr - Z0, ai = Zi, br = Zr + Z0, bi = Zi;
        const double bden = br * br + bi * bi;
        out[2 * f] = make_double2(Zr, Zi);
        out[2 * f + 1] = make_double2((ar * br + ai * bi) / bden, (ai * br - ar * bi) / bden);
    }
}

// x_f = 0 for the active slots f (grid (N / 256, B)); the others keep theirs
__global__ void k_zero_active(int N, double2 *__restrict__ x, const int *__restrict__ active) {
    const int f = blockIdx.y, i = blockIdx.x * blockDim.x + threadIdx.x;
    if (active[f] && i < N) x[(size_t)N * f + i] = make_double2(0.0, 0.0);
}

__global__ void k_init_ctl(int B, char *__restrict__ ctl, double bnorm, const int *__restrict__ active) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= B) return;
    char *c = ctl + 64 * f;
    double *red = reinterpret_cast<double *>(c);
    red[0] = 0.0;
    red[1] = bnorm;
    red[2] = 1.0;
    *reinterpret_cast<unsigned int *>(c + 24) = 0u;
    *reinterpret_cast<int *>(c + 28) = 0;
    *reinterpret_cast<int *>(c + 32) = active[f] ? 0 : 1;  // inactive slots count as converged
}

efie_status set_smem_attrs() {
    static bool done = false;
    if (done) return EFIE_OK;
    EFIE_CUDA(cudaFuncSetAttribute(k_panels, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPanelSmem));
    EFIE_CUDA(cudaFuncSetAttribute(k_diag_factor, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDiagSmem));
    EFIE_CUDA(cudaFuncSetAttribute(k_update_simt, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTwoTiles));
    done = true;
    return EFIE_OK;
}

}  // namespace

int efie_solve_nb() { return NB; }

efie_status efie_mixed_workspace(SolveWork &w, int N, int B, int kb_outer) {
    EFIE_TRY(set_smem_attrs());
    if (kb_outer != 64 && kb_outer != 128 && kb_outer != 256 && kb_outer != 512)
        return efie_fail(EFIE_ERR_ARGS, "LU panel width must be 64, 128, 256 or 512");
    w.kb_outer = kb_outer;
    w.N = N;
    w.B = B;
    w.ld = (N + 63) / 64 * 64;
    w.nblk = (N + NB - 1) / NB;
    w.pstride = 2 * (size_t)w.ld * N;
    w.dstride = 2 * (size_t)NB * NB * w.nblk;
    w.vstride = w.ld;
    const size_t pbytes = sizeof(float) * w.pstride * B;
    if (pbytes > w.planes.bytes) {
        EFIE_TRY(w.planes.reserve(pbytes));
        // the padding columns N .. ld-1 of every row stay zero (the triangular
        // solves' aligned loads read them); every other entry is written per batch
        if (w.ld > N)
            EFIE_CUDA(cudaMemset2D(w.planes.as<float>() + N, sizeof(float) * w.ld, 0, sizeof(float) * (w.ld - N),
                                   (size_t)2 * N * B));
    }
    EFIE_TRY(w.dinv.reserve(sizeof(float2) * w.dstride * B));
    EFIE_TRY(w.vec.reserve(sizeof(float2) * 3 * (size_t)w.vstride * B));
    EFIE_TRY(w.ctl.reserve(64 * (size_t)B + 64));
    EFIE_TRY(w.rpart.reserve(sizeof(double) * (size_t)B * ((N + 31) / 32)));
    w.mstride = (size_t)w.ld * w.nblk;
    EFIE_TRY(w.lmax.reserve(sizeof(float) * w.mstride * B));
    EFIE_TRY(w.umax.reserve(sizeof(float) * w.mstride * B));
    EFIE_TRY(w.active.reserve(sizeof(int) * B));
    EFIE_TRY(w.fsrc.reserve(sizeof(int) * B));
    w.fsrc_on = false;
    EFIE_TRY(efie_trsv_workspace(w));
    EFIE_TRY(efie_gemm_workspace(w));
    if (!w.hi) {
        int least = 0, greatest = 0;
        EFIE_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        EFIE_CUDA(cudaStreamCreateWithPriority(&w.hi, cudaStreamNonBlocking, greatest));
        EFIE_CUDA(cudaStreamCreateWithPriority(&w.lo, cudaStreamNonBlocking, least));
        for (cudaEvent_t *e : {&w.ev_start, &w.ev_panel, &w.ev_rest, &w.ev_hi})
            EFIE_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    }
    return EFIE_OK;
}

efie_status efie_mixed_factor_prepare(efie_ctx *ctx, SolveWork &w, const int *active_host) {
    cudaStream_t s = ctx->stream;
    EFIE_CUDA(cudaMemsetAsync(w.ctl.p, 0, 64 * (size_t)w.B, s));
    EFIE_CUDA(cudaMemcpyAsync(w.active.p, active_host, sizeof(int) * w.B, cudaMemcpyHostToDevice, s));
    return EFIE_OK;
}

efie_status efie_mixed_factor(efie_ctx *ctx, SolveWork &w, const void *Z, size_t zstride, const int *active_host) {
    int nact = 0;
    for (int f = 0; f < w.B; f++) nact += active_host[f] ? 1 : 0;
    EFIE_TRY(efie_mixed_factor_prepare(ctx, w, active_host));
    return efie_mixed_factor_launch(ctx, w, Z, zstride, nact);
}

namespace {

// Launches of a scope go to `s` (ctx->stream is the launch stream of every helper).
struct OnStream {
    efie_ctx *c;
    cudaStream_t old;
    OnStream(efie_ctx *ctx, cudaStream_t s) : c(ctx), old(ctx->stream) { c->stream = s; }
    ~OnStream() { c->stream = old; }
};

}  // namespace

// Two-level blocked LU with look-ahead.  Outer panel P = columns [K0, Kend)
// is factored by 64-wide diagonal blocks whose panel products and updates
// stay inside its L-shaped region (the panel chain F_P, latency bound).  Its
// deferred trailing update D_P (rows and columns >= Kend, K = Kend - K0) is
// split into the L-shaped strip of the next panel, D_P^next = rows
// [Kend, K1) x columns >= Kend and rows >= K1 x columns [Kend, K1)
// (K1 = Kend + KB), and the rest, D_P^rest = rows and columns >= K1.  The
// panel chain and D^next run on the high-priority stream; D^rest runs on the
// low-priority stream after F_P, so F_{P+1} overlaps D_P^rest (they touch
// disjoint parts of the matrix; D_P^next waits for D_{P-1}^rest, whose
// region contains it).
static int g_sym_lu_disabled = 0;
extern "C" void efie_debug_disable_symmetric_lu(int disable) { g_sym_lu_disabled = disable; }

efie_status efie_mixed_factor_launch(efie_ctx *ctx, SolveWork &w, const void *Z, size_t zstride, int nact) {
    cudaStream_t s0 = ctx->stream;
    KernelLog &log = ctx->log;
    const int N = w.N, ld = w.ld, B = w.B;
    float *planes = w.planes.as<float>();
    char *ctl = w.ctl.as<char>();
    const int *active = w.active.as<int>();
    dim3 tg((N + 31) / 32, (N + 31) / 32, B);
    size_t tok = 0;
    const bool sym = w.zsym && w.sym_lu && g_sym_lu_disabled != 1;
    if (!w.planes_from_assembly || !sym) {
        // the general LU reads the upper triangle of the planes too: from all of Z
        if (w.planes_from_assembly)
            for (int f = 0; f < B; f++)
                EFIE_TRY(efie_z_mirror(ctx, static_cast<double2 *>(const_cast<void *>(Z)) + zstride * f, N));
        tok = log.begin(s0);
        k_z_to_planes<<<tg, 256, 0, s0>>>(N, static_cast<const double2 *>(Z), zstride, planes, w.pstride, ld);
        EFIE_CUDA(cudaGetLastError());
        log.end(EFIE_K_PANEL, s0, tok, 24.0 * (double)N * N * nact);
    }
    float2 *dinv = w.dinv.as<float2>();
    EFIE_CUDA(cudaEventRecord(w.ev_start, s0));
    EFIE_CUDA(cudaStreamWaitEvent(w.hi, w.ev_start, 0));
    const int KB = w.kb_outer;
    // symmetric Z: every update keeps the lower part only (and the outer
    // panels' diagonal blocks); the diagonal blocks are factored from their
    // lower triangle and the row panel is formed from the column panel's
    // tiles, U[k.., j] = L_kk^-1 A[j, k..]^T, so that L and U follow from
    // the same (lower) data
    const bool symtri = sym && g_sym_lu_disabled != 2;
    bool rest_pending = false;   // ev_rest holds the record of the previous D^rest
    // with per-launch timing on, D^rest goes to the chain's stream too: the
    // launches run one at a time, so each pair of events brackets its kernel
    // alone instead of a kernel sharing the SMs with the other stream's
    cudaStream_t lo = log.timing ? w.hi : w.lo;
    const PackView ipl = efie_inpanel_view(w, true), ipu = efie_inpanel_view(w, false);
    {
        OnStream on(ctx, w.hi);
        cudaStream_t s = w.hi;
        for (int K0 = 0, P = 0; K0 < N; K0 += KB, P++) {
            const int Kend = std::min(N, K0 + KB), K1 = std::min(N, Kend + KB);
            // F_P: the panel chain; the panel kernel packs each 64-wide block
            // for the chain's two updates (K = 64).  With the lower-triangle
            // scheme a panel of 512 is factored as two halves: the chain of the
            // first half updates only the first half's columns, then one K = 256
            // update brings the second half's columns (every row below them) up
            // to date before its own chain -- the K = 64 updates read and write
            // a block of C once per 64 of K, so this cuts their C traffic by
            // about 40 % at the cost of one more pair of packs.
            const int H = (symtri && KB >= 512 && Kend - K0 > KB / 2) ? K0 + KB / 2 : Kend;
            for (int half = 0; half < 2; half++) {
                const int Hs = half == 0 ? K0 : H, He = half == 0 ? H : Kend;
                if (Hs >= He) break;
                for (int k = Hs; k < He; k += NB) {
                    const int bi = k / NB, kb = std::min(NB, N - k);
                    const int s1 = k + kb, rest = N - s1;
                    const bool inpanel = s1 < He;
                    tok = log.begin(s);
                    k_diag_factor<<<B, 256, kDiagSmem, s>>>(N, k, kb, bi, planes, w.pstride, ld, dinv, w.dstride, ctl,
                                                            active, sym ? (g_sym_lu_disabled == 3 ? 2 : 1) : 0);
                    if (rest > 0) {
                        dim3 pg((rest + NB - 1) / NB, sym ? 1 : 2, B);
                        k_panels<<<pg, 256, kPanelSmem, s>>>(N, k, kb, bi, planes, w.pstride, ld, dinv, w.dstride,
                                                             active, w.lmax.as<float>(), w.umax.as<float>(),
                                                             w.mstride, w.nblk, w.ipL.as<__half>(), w.ipU.as<__half>(),
                                                             ipl.stride, ipl.pitch, inpanel ? 1 : 0, sym ? 1 : 0, He);
                    }
                    EFIE_CUDA(cudaGetLastError());
                    log.end(EFIE_K_PANEL, s, tok, 0.0, rest > 0 ? 2 : 1);
                    if (inpanel && sym) {
                        // every row below the block, the (half) panel's remaining columns
                        EFIE_TRY(efie_gemm_update(ctx, w, s1, N, s1, He, k, k, kb, nact, ipl, ipu));
                    } else if (inpanel) {
                        // rows of this panel below the block, every column to the right
                        EFIE_TRY(efie_gemm_update(ctx, w, s1, He, s1, N, k, k, kb, nact, ipl, ipu));
                        // rows below the panel, the panel's remaining columns
                        EFIE_TRY(efie_gemm_update(ctx, w, He, N, s1, He, k, k, kb, nact, ipl.at(He - s1), ipu));
                    }
                }
                if (half == 0 && H < Kend) {
                    // the first half's contribution to the second half's columns,
                    // through this panel's staging (free: panel P - 2's D^rest,
                    // its last reader, finished before D_{P-1}^next)
                    PackView Lh, Uh;
                    EFIE_TRY(efie_pack_l(ctx, w, w.packL[P & 1], H, N, K0, H - K0, &Lh));
                    EFIE_TRY(efie_pack_u(ctx, w, w.packU[P & 1], H, Kend, K0, H - K0, &Uh));
                    EFIE_TRY(efie_gemm_update(ctx, w, H, N, H, Kend, K0, K0, H - K0, nact, Lh, Uh));
                }
            }
            if (Kend >= N) break;
            // L and U of the panel packed once (staging of this panel's parity)
            // for D_P^next and D_P^rest; D_P^rest finishes before panel P + 2's
            // packs, which follow D_{P+1}^next on this stream
            const int K = Kend - K0;
            PackView Lp, Up;
            EFIE_TRY(efie_pack_l(ctx, w, w.packL[P & 1], Kend, N, K0, K, &Lp));
            EFIE_TRY(efie_pack_u(ctx, w, w.packU[P & 1], Kend, N, K0, K, &Up));
            EFIE_CUDA(cudaEventRecord(w.ev_panel, s));
            // D_P^next on the critical stream, after D_{P-1}^rest
            if (rest_pending) EFIE_CUDA(cudaStreamWaitEvent(s, w.ev_rest, 0));
            if (symtri) {
                // the next panel's columns (its diagonal block in full)
                EFIE_TRY(efie_gemm_update(ctx, w, Kend, N, Kend, K1, K0, K0, K, nact, Lp, Up));
            } else {
                EFIE_TRY(efie_gemm_update(ctx, w, Kend, K1, Kend, N, K0, K0, K, nact, Lp, Up));
                EFIE_TRY(efie_gemm_update(ctx, w, K1, N, Kend, K1, K0, K0, K, nact, Lp.at(K1 - Kend), Up));
            }
            // D_P^rest on the low-priority stream, after F_P and the packs
            if (K1 < N) {
                OnStream on_lo(ctx, lo);
                EFIE_CUDA(cudaStreamWaitEvent(lo, w.ev_panel, 0));
                EFIE_TRY(efie_gemm_update(ctx, w, K1, N, K1, N, K0, K0, K, nact, Lp.at(K1 - Kend),
                                          Up.at(K1 - Kend), symtri ? KB : 0));
                EFIE_CUDA(cudaEventRecord(w.ev_rest, lo));
                rest_pending = true;
            }
        }
    }
    // join both streams back into the caller's stream
    EFIE_CUDA(cudaEventRecord(w.ev_hi, w.hi));
    EFIE_CUDA(cudaStreamWaitEvent(s0, w.ev_hi, 0));
    if (rest_pending) EFIE_CUDA(cudaStreamWaitEvent(s0, w.ev_rest, 0));
    return EFIE_OK;
}

efie_status efie_update_simt(efie_ctx *ctx, SolveWork &w, int r0, int r1, int c0, int c1, int kcol, int krow, int K,
                             int nact) {
    const int N = w.N;
    if (r1 <= r0 || c1 <= c0) return EFIE_OK;
    dim3 g((c1 - c0 + NB - 1) / NB, (r1 - r0 + NB - 1) / NB, w.B);
    size_t tok = ctx->log.begin(ctx->stream);
    k_update_simt<<<g, 256, kTwoTiles, ctx->stream>>>(N, r0, r1, c0, c1, kcol, krow, K, w.planes.as<float>(),
                                                      w.pstride, w.ld, w.active.as<int>());
    EFIE_CUDA(cudaGetLastError());
    ctx->log.end(EFIE_K_GEMM, ctx->stream, tok, 8.0 * (double)(r1 - r0) * (c1 - c0) * K * nact);
    return EFIE_OK;
}

efie_status efie_mixed_refine(efie_ctx *ctx, SolveWork &w, const void *Z, size_t zstride, const void *b, void *x,
                              double bnorm, double tol, int max_iter, const int *active_host, RefineResult *res) {
    cudaStream_t s = ctx->stream;
    KernelLog &log = ctx->log;
    const int N = w.N, B = w.B;
    char *ctl = w.ctl.as<char>();
    float2 *vec = w.vec.as<float2>();
    float2 *rf = vec, *y = vec + (size_t)w.vstride * B, *d = y + (size_t)w.vstride * B;
    int nact = 0;
    for (int f = 0; f < B; f++) nact += active_host[f] ? 1 : 0;
    const double zbytes = 16.0 * (double)N * N, lubytes = 8.0 * (double)N * N;
    size_t tok = log.begin(s);
    k_zero_active<<<dim3((N + 255) / 256, B), 256, 0, s>>>(N, static_cast<double2 *>(x), w.active.as<int>());
    k_init_ctl<<<(B + 63) / 64, 64, 0, s>>>(B, ctl, bnorm, w.active.as<int>());
    EFIE_CUDA(cudaGetLastError());
    log.end(EFIE_K_OTHER, s, tok, 0.0, 2);
    // initial residual r = V (x = 0) through the residual kernel keeps one code path
    dim3 rg((N + 31) / 32, B);
    tok = log.begin(s);
    k_residual<<<rg, 256, 0, s>>>(N, static_cast<const double2 *>(Z), zstride, static_cast<const double2 *>(x),
                                  static_cast<const double2 *>(b), rf, w.vstride, ctl, -1.0, nullptr,
                                  w.rpart.as<double>());
    EFIE_CUDA(cudaGetLastError());
    log.end(EFIE_K_RESIDUAL, s, tok, zbytes * nact);
    int it = 0;
    std::vector<char> hctl(64 * (size_t)B);
    bool all_done = false, failed = false;
    while (!all_done && !failed) {
        const int chunk = std::min(5, max_iter - it);
        if (chunk <= 0) break;
        for (int c = 0; c < chunk; c++) {
            const int epoch = ++w.epoch;
            tok = log.begin(s);
            EFIE_TRY(efie_trsv(ctx, w, true, rf, y, x, epoch));
            EFIE_TRY(efie_trsv(ctx, w, false, y, d, x, epoch));
            log.end(EFIE_K_TRSV, s, tok, lubytes * nact, 2);
            tok = log.begin(s);
            k_residual<<<rg, 256, 0, s>>>(N, static_cast<const double2 *>(Z), zstride,
                                          static_cast<const double2 *>(x), static_cast<const double2 *>(b), rf,
                                          w.vstride, ctl, tol, nullptr, w.rpart.as<double>());
            EFIE_CUDA(cudaGetLastError());
            log.end(EFIE_K_RESIDUAL, s, tok, zbytes * nact);
        }
        it += chunk;
        EFIE_CUDA(cudaMemcpyAsync(hctl.data(), ctl, 64 * (size_t)B, cudaMemcpyDeviceToHost, s));
        EFIE_CUDA(cudaStreamSynchronize(s));
        all_done = true;
        for (int f = 0; f < B; f++) {
            const char *c = hctl.data() + 64 * f;
            if (!active_host[f]) continue;
            if (*reinterpret_cast<const int *>(c + 36)) failed = true;
            if (!*reinterpret_cast<const int *>(c + 28)) all_done = false;
        }
    }
    EFIE_CUDA(cudaMemcpyAsync(hctl.data(), ctl, 64 * (size_t)B, cudaMemcpyDeviceToHost, s));
    EFIE_CUDA(cudaStreamSynchronize(s));
    res->iters = it;
    for (int f = 0; f < B; f++) {
        const char *c = hctl.data() + 64 * f;
        res->relres[f] = reinterpret_cast<const double *>(c)[2];
        res->converged[f] = *reinterpret_cast<const int *>(c + 28) != 0;
        res->err[f] = *reinterpret_cast<const int *>(c + 36);
    }
    return EFIE_OK;
}

efie_status efie_true_residual(efie_ctx *ctx, SolveWork &w, const void *Z, size_t zstride, const void *x,
                               const void *b, double tol, void *rout, int nact) {
    cudaStream_t s = ctx->stream;
    dim3 rg((w.N + 31) / 32, w.B);
    size_t tok = ctx->log.begin(s);
    k_residual<<<rg, 256, 0, s>>>(w.N, static_cast<const double2 *>(Z), zstride, static_cast<const double2 *>(x),
                                  static_cast<const double2 *>(b), w.vec.as<float2>(), w.vstride, w.ctl.as<char>(),
                                  tol, static_cast<double2 *>(rout), w.rpart.as<double>());
    EFIE_CUDA(cudaGetLastError());
    ctx->log.end(EFIE_K_RESIDUAL, s, tok, 16.0 * (double)w.N * w.N * nact);
    return EFIE_OK;
}

efie_status efie_residual_finish(efie_ctx *ctx, SolveWork &w, const void *y, const void *b, double tol, void *rout,
                                 int nact) {
    cudaStream_t s = ctx->stream;
    size_t tok = ctx->log.begin(s);
    k_resid_finish<<<dim3((w.N + 255) / 256, w.B), 256, 0, s>>>(
        w.N, static_cast<const double2 *>(y), static_cast<const double2 *>(b), w.vec.as<float2>(), w.vstride,
        w.ctl.as<char>(), tol, static_cast<double2 *>(rout), w.rpart.as<double>());
    EFIE_CUDA(cudaGetLastError());
    ctx->log.end(EFIE_K_RESIDUAL, s, tok, 0.0);
    return EFIE_OK;
}

efie_status efie_refine_init(efie_ctx *ctx, SolveWork &w, void *x, double bnorm, bool zero_x) {
    cudaStream_t s = ctx->stream;
    const int N = w.N, B = w.B;
    size_t tok = ctx->log.begin(s);
    if (zero_x)
        k_zero_active<<<dim3((N + 255) / 256, B), 256, 0, s>>>(N, static_cast<double2 *>(x), w.active.as<int>());
    k_init_ctl<<<(B + 63) / 64, 64, 0, s>>>(B, w.ctl.as<char>(), bnorm, w.active.as<int>());
    EFIE_CUDA(cudaGetLastError());
    ctx->log.end(EFIE_K_OTHER, s, tok, 0.0, zero_x ? 2 : 1);
    return EFIE_OK;
}

namespace {
__global__ void k_interp_guess(int N, double2 *__restrict__ x, const double2 *__restrict__ xs, GuessSpec g) {
    const int f = blockIdx.y, i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double2 v = make_double2(0.0, 0.0);
#pragma unroll
    for (int t = 0; t < 3; t++) {
        if (g.idx[t][f] < 0) continue;
        const double2 a = xs[(size_t)N * g.idx[t][f] + i];
        v.x += g.w[t][f] * a.x;
        v.y += g.w[t][f] * a.y;
    }
    x[(size_t)N * f + i] = v;
}
}  // namespace

efie_status efie_interp_guess(efie_ctx *ctx, int N, int n, void *x, const void *xs, const GuessSpec &g) {
    if (n <= 0) return EFIE_OK;
    size_t tok = ctx->log.begin(ctx->stream);
    k_interp_guess<<<dim3((N + 255) / 256, n), 256, 0, ctx->stream>>>(N, static_cast<double2 *>(x),
                                                                     static_cast<const double2 *>(xs), g);
    EFIE_CUDA(cudaGetLastError());
    ctx->log.end(EFIE_K_OTHER, ctx->stream, tok, 0.0);
    return EFIE_OK;
}

efie_status efie_port_reduce(efie_ctx *ctx, int N, int B, const void *x, const double *wport, int model, int pe,
                             int ge, double V0, double Z0, void *out) {
    size_t tok = ctx->log.begin(ctx->stream);
    k_port<<<B, 1024, 0, ctx->stream>>>(N, static_cast<const double2 *>(x), wport, model, pe, ge, V0, Z0,
                                         static_cast<double2 *>(out));
    EFIE_CUDA(cudaGetLastError());
    ctx->log.end(EFIE_K_OTHER, ctx->stream, tok, 0.0);
    return EFIE_OK;
}
