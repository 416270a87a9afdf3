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

#include "efie_internal.h"
#include "solve.h"

namespace {

constexpr int NB = 64;   // diagonal block size of the LU and the triangular solves
constexpr size_t kTwoTiles = sizeof(float2) * 2 * NB * (NB + 1);

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
// Diagonal block bi of every frequency (blockIdx.x = f): unblocked LU without
// pivoting of A[k:k+kb, k:k+kb] and the inverses of its unit-lower L and upper
// U factors (kept for the panel products and the triangular solves).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_diag_factor(int N, int k, int kb, int bi, float *__restrict__ planes,
                                                      size_t pstride, int ld, float2 *__restrict__ dinv,
                                                      size_t dstride, char *__restrict__ ctl,
                                                      const int *__restrict__ active) {
    const int f = blockIdx.x;
    if (!active[f]) return;
    extern __shared__ float2 dyn[];
    float2(*a)[NB + 1] = reinterpret_cast<float2(*)[NB + 1]>(dyn);
    float2(*w)[NB + 1] = reinterpret_cast<float2(*)[NB + 1]>(dyn + NB * (NB + 1));
    float *Ar = planes + pstride * f, *Ai = Ar + (size_t)ld * N;
    float2 *Linv = dinv + dstride * f + (size_t)bi * 2 * NB * NB, *Uinv = Linv + NB * NB;
    int *err = reinterpret_cast<int *>(ctl + 64 * f + 36);
    const int tid = threadIdx.x;
    for (int e = tid; e < NB * NB; e += 1024) {
        const int i = e / NB, j = e % NB;
        float2 v = make_float2(0.f, 0.f);
        if (i < kb && j < kb) v = make_float2(Ar[(size_t)(k + i) * ld + k + j], Ai[(size_t)(k + i) * ld + k + j]);
        else if (i == j) v = make_float2(1.f, 0.f);  // pad to identity
        a[i][j] = v;
    }
    __syncthreads();
    for (int j = 0; j < NB - 1; j++) {
        const float2 p = a[j][j];
        const float den = p.x * p.x + p.y * p.y;
        if (tid == 0 && !(den > 0.f)) atomicExch(err, 1);
        const float2 pinv = make_float2(p.x / den, -p.y / den);
        if (tid > j && tid < NB) a[tid][j] = cmulf(a[tid][j], pinv);
        __syncthreads();
        for (int e = tid; e < NB * NB; e += 1024) {
            const int i = e / NB, c = e % NB;
            if (i > j && c > j) {
                const float2 l = a[i][j], u = a[j][c];
                a[i][c].x -= l.x * u.x - l.y * u.y;
                a[i][c].y -= l.x * u.y + l.y * u.x;
            }
        }
        __syncthreads();
    }
    if (tid == 0) {
        const float2 p = a[NB - 1][NB - 1];
        if (!(p.x * p.x + p.y * p.y > 0.f)) atomicExch(err, 1);
    }
    for (int e = tid; e < NB * NB; e += 1024) {
        const int i = e / NB, j = e % NB;
        if (i < kb && j < kb) {
            Ar[(size_t)(k + i) * ld + k + j] = a[i][j].x;
            Ai[(size_t)(k + i) * ld + k + j] = a[i][j].y;
        }
    }
    // Linv: unit lower; column c by forward substitution, 16 threads per column
    const int c = tid >> 4, sub = tid & 15;
    for (int i = 0; i < NB; i++) {
        float2 s = make_float2(0.f, 0.f);
        for (int j = c + sub; j < i; j += 16) {
            const float2 l = a[i][j], x = w[j][c];
            s.x += l.x * x.x - l.y * x.y;
            s.y += l.x * x.y + l.y * x.x;
        }
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) {
            s.x += __shfl_xor_sync(0xffffffffu, s.x, o, 16);
            s.y += __shfl_xor_sync(0xffffffffu, s.y, o, 16);
        }
        if (sub == 0) w[i][c] = (i < c) ? make_float2(0.f, 0.f) : (i == c ? make_float2(1.f, 0.f) : make_float2(-s.x, -s.y));
        __syncthreads();
    }
    for (int e = tid; e < NB * NB; e += 1024) Linv[e] = w[e / NB][e % NB];
    __syncthreads();
    // Uinv: upper; column c by backward substitution
    for (int i = NB - 1; i >= 0; i--) {
        float2 s = make_float2(0.f, 0.f);
        for (int j = i + 1 + sub; j <= c; j += 16) {
            const float2 u = a[i][j], x = w[j][c];
            s.x += u.x * x.x - u.y * x.y;
            s.y += u.x * x.y + u.y * x.x;
        }
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) {
            s.x += __shfl_xor_sync(0xffffffffu, s.x, o, 16);
            s.y += __shfl_xor_sync(0xffffffffu, s.y, o, 16);
        }
        if (sub == 0) {
            float2 r = make_float2(0.f, 0.f);
            if (i <= c) {
                const float2 d = a[i][i];
                const float den = d.x * d.x + d.y * d.y;
                const float2 rhs = (i == c) ? make_float2(1.f - s.x, -s.y) : make_float2(-s.x, -s.y);
                r = make_float2((rhs.x * d.x + rhs.y * d.y) / den, (rhs.y * d.x - rhs.x * d.y) / den);
            }
            w[i][c] = r;
        }
        __syncthreads();
    }
    for (int e = tid; e < NB * NB; e += 1024) Uinv[e] = w[e / NB][e % NB];
}

// ---------------------------------------------------------------------------
// Panels: U12 = Linv * A12 (row panel) and L21 = A21 * Uinv (column panel).
// One 64x64 tile per CTA, in place.  blockIdx.y: 0 row panel, 1 column panel;
// blockIdx.z: frequency.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_panels(int N, int k, int kb, int bi, float *__restrict__ planes,
                                                size_t pstride, int ld, const float2 *__restrict__ dinv,
                                                size_t dstride, const int *__restrict__ active) {
    const int f = blockIdx.z;
    if (!active[f]) return;
    extern __shared__ float2 dyn[];
    float2(*M)[NB + 1] = reinterpret_cast<float2(*)[NB + 1]>(dyn);               // the inverse
    float2(*T)[NB + 1] = reinterpret_cast<float2(*)[NB + 1]>(dyn + NB * (NB + 1));  // the panel tile
    float *Ar = planes + pstride * f, *Ai = Ar + (size_t)ld * N;
    const float2 *Linv = dinv + dstride * f + (size_t)bi * 2 * NB * NB, *Uinv = Linv + NB * NB;
    const int tid = threadIdx.x;
    const bool rowp = blockIdx.y == 0;
    const int off = k + kb + blockIdx.x * NB;
    if (off >= N) return;
    const int ext = min(NB, N - off);
    const float2 *inv = rowp ? Linv : Uinv;
    for (int e = tid; e < NB * NB; e += 256) M[e / NB][e % NB] = inv[e];
    for (int e = tid; e < NB * NB; e += 256) {
        const int i = e / NB, j = e % NB;
        float2 v = make_float2(0.f, 0.f);
        if (rowp) {
            if (i < kb && j < ext) v = make_float2(Ar[(size_t)(k + i) * ld + off + j], Ai[(size_t)(k + i) * ld + off + j]);
        } else {
            if (i < ext && j < kb) v = make_float2(Ar[(size_t)(off + i) * ld + k + j], Ai[(size_t)(off + i) * ld + k + j]);
        }
        T[i][j] = v;
    }
    __syncthreads();
    const int r0 = (tid >> 4) * 4, c0 = (tid & 15) * 4;
    float2 acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) acc[a][b] = make_float2(0.f, 0.f);
    for (int q = 0; q < NB; q++) {
        float2 x[4], y[4];
#pragma unroll
        for (int a = 0; a < 4; a++) {
            x[a] = rowp ? M[r0 + a][q] : T[r0 + a][q];
            y[a] = rowp ? T[q][c0 + a] : M[q][c0 + a];
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
            const int i = r0 + a, j = c0 + b;
            if (rowp) {
                if (i < kb && j < ext) {
                    Ar[(size_t)(k + i) * ld + off + j] = acc[a][b].x;
                    Ai[(size_t)(k + i) * ld + off + j] = acc[a][b].y;
                }
            } else {
                if (i < ext && j < kb) {
                    Ar[(size_t)(off + i) * ld + k + j] = acc[a][b].x;
                    Ai[(size_t)(off + i) * ld + k + j] = acc[a][b].y;
                }
            }
        }
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
                                                  double tol, double2 *__restrict__ routb) {
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
    if (threadIdx.x == 0) {
        double q = 0.0;
        for (int i = 0; i < 32; i++) q += sq[i];
        atomicAdd(red, q);
        __threadfence();
        const unsigned int done = atomicAdd(counter, 1u);
        last = (done == gridDim.x - 1);
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        const double rr = sqrt(*((volatile double *)red));
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

__global__ void k_fill_c128(size_t n, double2 *__restrict__ dst, double2 v) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = v;
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
    EFIE_CUDA(cudaFuncSetAttribute(k_diag_factor, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTwoTiles));
    EFIE_CUDA(cudaFuncSetAttribute(k_panels, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTwoTiles));
    EFIE_CUDA(cudaFuncSetAttribute(k_update_simt, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTwoTiles));
    done = true;
    return EFIE_OK;
}

}  // namespace

int efie_solve_nb() { return NB; }

efie_status efie_mixed_workspace(SolveWork &w, int N, int B, int kb_outer) {
    EFIE_TRY(set_smem_attrs());
    if (kb_outer != 64 && kb_outer != 128 && kb_outer != 256)
        return efie_fail(EFIE_ERR_ARGS, "LU panel width must be 64, 128 or 256");
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
        EFIE_CUDA(cudaMemset(w.planes.p, 0, pbytes));  // padding columns stay zero
    }
    EFIE_TRY(w.dinv.reserve(sizeof(float2) * w.dstride * B));
    EFIE_TRY(w.vec.reserve(sizeof(float2) * 3 * (size_t)w.vstride * B));
    EFIE_TRY(w.ctl.reserve(64 * (size_t)B + 64));
    EFIE_TRY(w.active.reserve(sizeof(int) * B));
    EFIE_TRY(efie_trsv_workspace(w));
    return EFIE_OK;
}

efie_status efie_mixed_factor(efie_ctx *ctx, SolveWork &w, const void *Z, size_t zstride, const int *active_host) {
    cudaStream_t s = ctx->stream;
    KernelLog &log = ctx->log;
    const int N = w.N, ld = w.ld, B = w.B;
    float *planes = w.planes.as<float>();
    char *ctl = w.ctl.as<char>();
    int nact = 0;
    for (int f = 0; f < B; f++) nact += active_host[f] ? 1 : 0;
    EFIE_CUDA(cudaMemsetAsync(w.ctl.p, 0, 64 * (size_t)B, s));
    EFIE_CUDA(cudaMemcpyAsync(w.active.p, active_host, sizeof(int) * B, cudaMemcpyHostToDevice, s));
    const int *active = w.active.as<int>();
    dim3 tg((N + 31) / 32, (N + 31) / 32, B);
    size_t tok = log.begin(s);
    k_z_to_planes<<<tg, 256, 0, s>>>(N, static_cast<const double2 *>(Z), zstride, planes, w.pstride, ld);
    EFIE_CUDA(cudaGetLastError());
    log.end(EFIE_K_PANEL, s, tok, 24.0 * (double)N * N * nact);
    float2 *dinv = w.dinv.as<float2>();
    // Two-level blocking: outer panels of KB columns are factored with 64-wide
    // diagonal blocks whose updates stay inside the panel's L-shaped region;
    // the rest of the trailing matrix gets one update with K = KB.
    const int KB = w.kb_outer;
    for (int K0 = 0; K0 < N; K0 += KB) {
        const int Kend = std::min(N, K0 + KB);
        for (int k = K0; k < Kend; k += NB) {
            const int bi = k / NB, kb = std::min(NB, N - k);
            const int s1 = k + kb, rest = N - s1;
            tok = log.begin(s);
            k_diag_factor<<<B, 1024, kTwoTiles, s>>>(N, k, kb, bi, planes, w.pstride, ld, dinv, w.dstride, ctl,
                                                     active);
            if (rest > 0) {
                dim3 pg((rest + NB - 1) / NB, 2, B);
                k_panels<<<pg, 256, kTwoTiles, s>>>(N, k, kb, bi, planes, w.pstride, ld, dinv, w.dstride, active);
            }
            EFIE_CUDA(cudaGetLastError());
            log.end(EFIE_K_PANEL, s, tok, 0.0, rest > 0 ? 2 : 1);
            if (s1 < Kend) {
                // rows of this panel below the block, every column to the right
                EFIE_TRY(efie_gemm_update(ctx, w, s1, Kend, s1, N, k, k, kb, nact));
                // rows below the panel, the panel's remaining columns
                EFIE_TRY(efie_gemm_update(ctx, w, Kend, N, s1, Kend, k, k, kb, nact));
            }
        }
        // the deferred trailing update with the whole panel
        EFIE_TRY(efie_gemm_update(ctx, w, Kend, N, Kend, N, K0, K0, Kend - K0, nact));
    }
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
    k_fill_c128<<<(unsigned)(((size_t)N * B + 255) / 256), 256, 0, s>>>((size_t)N * B, static_cast<double2 *>(x),
                                                                        make_double2(0.0, 0.0));
    k_init_ctl<<<(B + 63) / 64, 64, 0, s>>>(B, ctl, bnorm, w.active.as<int>());
    EFIE_CUDA(cudaGetLastError());
    log.end(EFIE_K_OTHER, s, tok, 0.0, 2);
    // initial residual r = V (x = 0) through the residual kernel keeps one code path
    dim3 rg((N + 31) / 32, B);
    tok = log.begin(s);
    k_residual<<<rg, 256, 0, s>>>(N, static_cast<const double2 *>(Z), zstride, static_cast<const double2 *>(x),
                                  static_cast<const double2 *>(b), rf, w.vstride, ctl, -1.0, nullptr);
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
                                          w.vstride, ctl, tol, nullptr);
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
                                  tol, static_cast<double2 *>(rout));
    EFIE_CUDA(cudaGetLastError());
    ctx->log.end(EFIE_K_RESIDUAL, s, tok, 16.0 * (double)w.N * w.N * nact);
    return EFIE_OK;
}

efie_status efie_refine_init(efie_ctx *ctx, SolveWork &w, void *x, double bnorm) {
    cudaStream_t s = ctx->stream;
    const int N = w.N, B = w.B;
    size_t tok = ctx->log.begin(s);
    k_fill_c128<<<(unsigned)(((size_t)N * B + 255) / 256), 256, 0, s>>>((size_t)N * B, static_cast<double2 *>(x),
                                                                        make_double2(0.0, 0.0));
    k_init_ctl<<<(B + 63) / 64, 64, 0, s>>>(B, w.ctl.as<char>(), bnorm, w.active.as<int>());
    EFIE_CUDA(cudaGetLastError());
    ctx->log.end(EFIE_K_OTHER, s, tok, 0.0, 2);
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
