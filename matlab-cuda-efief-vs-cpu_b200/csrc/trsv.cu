// Triangular solves with the complex64 LU factors (row-major FP32 planes).
//
// One persistent cooperative grid per solve; CTA c owns block rows
// c, c + grid, ...  Block row b needs the solution blocks of every block it
// depends on (j < b for L, j > b for U); each dependency is a flag written
// with a release fence by the owning CTA and read with a bounded wait.
// Everything that does not depend on a flag is loaded before the wait: the
// inverse of the diagonal block (to shared memory) and the next L/U tile (to
// registers), so the critical path per block is the flag round trip, one
// 64-entry vector load and the 64x64 products.
#include "efie_internal.h"
#include "solve.h"

namespace {

constexpr int NB = 64;
constexpr int DS = NB + 1;  // padded row stride of the diagonal inverse in shared memory

__device__ __forceinline__ bool wait_flag(const volatile int *flag, int epoch, int *err) {
    long long spins = 0;
    while (*flag != epoch) {
        if (++spins > (1ll << 24)) {  // give up after ~1 s: record, let every waiter return
            atomicExch(err, 2);
            return false;
        }
        if (*((volatile int *)err)) return false;
        __nanosleep(32);
    }
    __threadfence();
    return true;
}

// 16 consecutive complex entries of one row of the planes (zeros past `rows`).
__device__ __forceinline__ void load_tile_row(float4 (&t)[8], const float *Ar, const float *Ai, size_t off,
                                              bool valid) {
    if (valid) {
        const float4 *pr = reinterpret_cast<const float4 *>(Ar + off);
        const float4 *pi = reinterpret_cast<const float4 *>(Ai + off);
#pragma unroll
        for (int i = 0; i < 4; i++) {
            t[i] = __ldg(pr + i);
            t[4 + i] = __ldg(pi + i);
        }
    } else {
#pragma unroll
        for (int i = 0; i < 8; i++) t[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

__device__ __forceinline__ float2 dot16(const float4 (&t)[8], const float2 *y) {
    const float *re = reinterpret_cast<const float *>(t);
    const float *im = re + 16;
    float2 s = make_float2(0.f, 0.f);
#pragma unroll
    for (int c = 0; c < 16; c++) {
        const float2 v = y[c];
        s.x += re[c] * v.x - im[c] * v.y;
        s.y += re[c] * v.y + im[c] * v.x;
    }
    return s;
}

template <bool LOWER>
__global__ void __launch_bounds__(256) k_trsv(int N, int nblk, const float *__restrict__ Ar,
                                              const float *__restrict__ Ai, int ld, const float2 *__restrict__ dinv,
                                              const float2 *__restrict__ rhs, float2 *out, double2 *__restrict__ x,
                                              int *flags, int epoch, int *err, const int *__restrict__ skip) {
    if (*skip) return;  // refinement already converged
    __shared__ float2 Ds[NB * DS];
    __shared__ float2 acc[NB];
    __shared__ float2 yj[NB];
    __shared__ float2 part[4][NB];
    __shared__ int ok;
    const int tid = threadIdx.x;
    const int row = tid & 63, quarter = tid >> 6;
    for (int it = blockIdx.x; it < nblk; it += gridDim.x) {
        const int b = LOWER ? it : nblk - 1 - it;
        const int r0 = b * NB;
        const int rows = min(NB, N - r0);
        const bool rvalid = row < rows;
        // independent of every flag: the diagonal inverse and the right-hand side
        const float2 *D = dinv + (size_t)b * 2 * NB * NB + (LOWER ? 0 : NB * NB);
        for (int e = tid; e < NB * NB; e += 256) Ds[(e >> 6) * DS + (e & 63)] = __ldg(D + e);
        if (tid < NB) acc[tid] = (tid < rows) ? rhs[r0 + tid] : make_float2(0.f, 0.f);
        if (tid == 0) ok = 1;
        const int jbeg = LOWER ? 0 : b + 1, jend = LOWER ? b : nblk;
        const size_t rowoff = (size_t)(r0 + (rvalid ? row : 0)) * ld + quarter * 16;
        float4 cur[8];
        if (jbeg < jend) load_tile_row(cur, Ar, Ai, rowoff + (size_t)jbeg * NB, rvalid);
        __syncthreads();
        for (int jb = jbeg; jb < jend; jb++) {
            float4 nxt[8];
            if (jb + 1 < jend) load_tile_row(nxt, Ar, Ai, rowoff + (size_t)(jb + 1) * NB, rvalid);
            if (tid == 0 && !wait_flag(flags + jb, epoch, err)) ok = 0;
            __syncthreads();
            if (!ok) return;
            // written by another CTA of this grid: read through L2 only
            if (tid < NB) yj[tid] = (jb * NB + tid < N) ? __ldcg(out + jb * NB + tid) : make_float2(0.f, 0.f);
            __syncthreads();
            part[quarter][row] = dot16(cur, yj + quarter * 16);
            __syncthreads();
            if (tid < NB) {
                float2 t = acc[tid];
                t.x -= part[0][tid].x + part[1][tid].x + part[2][tid].x + part[3][tid].x;
                t.y -= part[0][tid].y + part[1][tid].y + part[2][tid].y + part[3][tid].y;
                acc[tid] = t;
            }
            if (jb + 1 < jend) {
#pragma unroll
                for (int i = 0; i < 8; i++) cur[i] = nxt[i];
            }
        }
        __syncthreads();
        // y_b = inv(diagonal block) * acc
        {
            const float2 *drow = Ds + row * DS + quarter * 16;
            float2 s = make_float2(0.f, 0.f);
#pragma unroll
            for (int c = 0; c < 16; c++) {
                const float2 m = drow[c], v = acc[quarter * 16 + c];
                s.x += m.x * v.x - m.y * v.y;
                s.y += m.x * v.y + m.y * v.x;
            }
            part[quarter][row] = s;
        }
        __syncthreads();
        if (tid < rows) {
            float2 t;
            t.x = part[0][tid].x + part[1][tid].x + part[2][tid].x + part[3][tid].x;
            t.y = part[0][tid].y + part[1][tid].y + part[2][tid].y + part[3][tid].y;
            __stcg(out + r0 + tid, t);
            if (!LOWER) {
                double2 xv = x[r0 + tid];
                xv.x += (double)t.x;
                xv.y += (double)t.y;
                x[r0 + tid] = xv;
            }
        }
        __threadfence();
        __syncthreads();
        if (tid == 0) atomicExch(flags + b, epoch);
    }
}

}  // namespace

efie_status efie_trsv(efie_ctx *ctx, SolveWork &w, bool lower, const float2 *rhs, float2 *out, void *x, int *flags,
                      int epoch, int *err, const int *skip) {
    int grid = std::min(w.nblk, ctx->num_sms);
    const float *Ar = w.planes.as<float>(), *Ai = Ar + (size_t)w.ld * w.N;
    const float2 *dinv = w.dinv.as<float2>();
    double2 *xd = static_cast<double2 *>(x);
    void *args[] = {(void *)&w.N, (void *)&w.nblk, (void *)&Ar, (void *)&Ai, (void *)&w.ld, (void *)&dinv,
                    (void *)&rhs, (void *)&out, (void *)&xd, (void *)&flags, (void *)&epoch, (void *)&err,
                    (void *)&skip};
    const void *fn = lower ? (const void *)k_trsv<true> : (const void *)k_trsv<false>;
    EFIE_CUDA(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(256), args, 0, ctx->stream));
    return EFIE_OK;
}
