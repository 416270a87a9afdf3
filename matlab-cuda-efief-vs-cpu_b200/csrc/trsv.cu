// Triangular solves with the complex64 LU factors of a batch of frequencies.
//
// One persistent cooperative grid per solve covers every (block row,
// frequency) item; item i = o * B + f (o = block order: b for L, nblk-1-b
// for U) goes to CTA i mod G, so each CTA walks its items in increasing o and
// every dependency of an item sits earlier in some CTA's queue (no deadlock
// while all CTAs are resident, which the cooperative launch guarantees).
//
// Progress is published per (direction, frequency) as a 64-bit counter
// (epoch << 32 | blocks done) replicated once per CTA on its own 64-byte
// line: the CTA that finishes a block raises every replica with atomicMax,
// and a waiting CTA polls only its own replica, so no line is polled by more
// than one CTA.  Waits are bounded and abort on the frequency's error flag.
// Everything that does not depend on a counter is loaded before the wait:
// the inverse of the diagonal block (to shared memory) and the next L/U tile
// (to registers).
#include <algorithm>

#include "efie_internal.h"
#include "solve.h"

namespace {

constexpr int NB = 64;
constexpr int DS = NB + 1;    // padded row stride of the diagonal inverse in shared memory
constexpr int LINE = 8;       // u64 per 64-byte progress line

// Limits of the bounded waits, per device.  d_wait_spins: polls before a
// wait gives up (2^23, about a second).  d_wait_offset: added to every wait
// target; nonzero only under efie_debug_set_wait_test, where it makes every
// target unreachable (a count no block ever publishes) so that tests can make
// the waits run out on purpose.
__device__ long long d_wait_spins = 1ll << 23;
__device__ unsigned long long d_wait_offset = 0;

// Wait until the counter reaches `target`; returns the observed value (0 on
// timeout or error, after which every waiter returns).
__device__ __forceinline__ unsigned long long wait_progress(const volatile unsigned long long *ctr,
                                                            unsigned long long target, const volatile int *err) {
    long long spins = 0;
    const long long limit = d_wait_spins;
    target += d_wait_offset;
    unsigned long long v;
    while ((v = *ctr) < target) {
        if (++spins > limit) {  // give up: record, let every waiter return
            atomicExch((int *)err, 2);
            return 0;
        }
        if ((spins & 63) == 0 && *err) return 0;
        __nanosleep(40);
    }
    __threadfence();
    return v;
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
__global__ void __launch_bounds__(256) k_trsv(int N, int nblk, int B, const float *__restrict__ planes, size_t pstride,
                                              int ld, const float2 *__restrict__ dinv, size_t dstride,
                                              const float2 *__restrict__ rhsb, float2 *outb, int vstride,
                                              double2 *__restrict__ xb, unsigned long long *prog, int epoch,
                                              char *ctl, const int *__restrict__ active) {
    __shared__ float2 Ds[NB * DS];
    __shared__ float2 acc[NB];
    __shared__ int avail_sh;
    __shared__ float2 part[4][NB];
    __shared__ int ok;
    const int tid = threadIdx.x;
    const int row = tid & 63, quarter = tid >> 6;
    const int G = gridDim.x;
    const unsigned long long tag = (unsigned long long)(unsigned)epoch << 32;
    const int dir = LOWER ? 0 : 1;
    const int items = nblk * B;
    for (int it = blockIdx.x; it < items; it += G) {
        const int o = it / B, f = it - o * B;
        if (!active[f]) continue;
        const char *c = ctl + 64 * f;
        if (*reinterpret_cast<const volatile int *>(c + 32)) continue;  // converged: skip the whole frequency
        const volatile int *err = reinterpret_cast<const volatile int *>(c + 36);
        const int b = LOWER ? o : nblk - 1 - o;
        const float *Ar = planes + pstride * f, *Ai = Ar + (size_t)ld * N;
        const float2 *rhs = rhsb + (size_t)vstride * f;
        float2 *out = outb + (size_t)vstride * f;
        unsigned long long *myctr = prog + ((size_t)(dir * B + f) * G + blockIdx.x) * LINE;
        const int r0 = b * NB;
        const int rows = min(NB, N - r0);
        const bool rvalid = row < rows;
        // independent of every counter: the diagonal inverse and the right-hand side
        const float2 *D = dinv + dstride * f + (size_t)b * 2 * NB * NB + (LOWER ? 0 : NB * NB);
        for (int e = tid; e < NB * NB; e += 256) Ds[(e >> 6) * DS + (e & 63)] = __ldg(D + e);
        if (tid < NB) acc[tid] = (tid < rows) ? rhs[r0 + tid] : make_float2(0.f, 0.f);
        if (tid == 0) ok = 1;
        // dependencies in solve order: L needs blocks 0..b-1, U needs blocks nblk-1..b+1
        const int ndep = o;
        const size_t rowoff = (size_t)(r0 + (rvalid ? row : 0)) * ld + quarter * 16;
        float4 cur[8];
        if (ndep > 0) {
            const int jb0 = LOWER ? 0 : nblk - 1;
            load_tile_row(cur, Ar, Ai, rowoff + (size_t)jb0 * NB, rvalid);
        }
        if (tid == 0) avail_sh = 0;
        __syncthreads();
        // each thread keeps its quarter-row dot product in registers across the
        // dependencies; the CTA synchronises only when it has to wait for a block
        // that is not published yet (one observed count can cover many blocks)
        float2 sdot = make_float2(0.f, 0.f);
        int avail = 0;
        for (int q = 0; q < ndep; q++) {
            const int jb = LOWER ? q : nblk - 1 - q;
            float4 nxt[8];
            if (q + 1 < ndep) load_tile_row(nxt, Ar, Ai, rowoff + (size_t)(LOWER ? jb + 1 : jb - 1) * NB, rvalid);
            if (q >= avail) {
                if (tid == 0) {
                    const unsigned long long v = wait_progress(myctr, tag | (unsigned long long)(q + 1), err);
                    if (!v) ok = 0;
                    avail_sh = (int)(v & 0xffffffffull);
                }
                __syncthreads();
                if (!ok) return;
                avail = avail_sh;
            }
            // block jb of the solution: written by another CTA and published
            // before `avail` was read, then never changed in this launch, so the
            // (L1-cached) loads cannot see a stale line; a 64-entry block covers
            // whole 128-byte lines
            float2 y16[16];
            const float2 *ysrc = out + jb * NB + quarter * 16;
#pragma unroll
            for (int c = 0; c < 16; c++)
                y16[c] = (jb * NB + quarter * 16 + c < N) ? ysrc[c] : make_float2(0.f, 0.f);
            const float2 t = dot16(cur, y16);
            sdot.x += t.x;
            sdot.y += t.y;
            if (q + 1 < ndep) {
#pragma unroll
                for (int i = 0; i < 8; i++) cur[i] = nxt[i];
            }
        }
        part[quarter][row] = sdot;
        __syncthreads();
        if (tid < NB) {
            float2 t = acc[tid];
            t.x -= part[0][tid].x + part[1][tid].x + part[2][tid].x + part[3][tid].x;
            t.y -= part[0][tid].y + part[1][tid].y + part[2][tid].y + part[3][tid].y;
            acc[tid] = t;
        }
        __syncthreads();
        // y_b = inv(diagonal block) * acc
        {
            const float2 *drow = Ds + row * DS + quarter * 16;
            float2 s = make_float2(0.f, 0.f);
#pragma unroll
            for (int cc = 0; cc < 16; cc++) {
                const float2 m = drow[cc], v = acc[quarter * 16 + cc];
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
                double2 *x = xb + (size_t)N * f;
                double2 xv = x[r0 + tid];
                xv.x += (double)t.x;
                xv.y += (double)t.y;
                x[r0 + tid] = xv;
            }
        }
        __threadfence();
        __syncthreads();
        // publish: o + 1 blocks of (dir, f) are done, on every CTA's replica
        const unsigned long long v = tag | (unsigned long long)(o + 1);
        unsigned long long *base = prog + (size_t)(dir * B + f) * G * LINE;
        for (int t = tid; t < G; t += 256) atomicMax(base + (size_t)t * LINE, v);
    }
}

}  // namespace

// Test hook (process-wide, on the current device): every later triangular
// solve waits for a count that is never published and gives up after `spins`
// polls (enable = 1), or the production limits come back (enable = 0).
extern "C" efie_status efie_debug_set_wait_test(int32_t enable, int64_t spins) {
    const long long lim = enable ? (long long)std::max<int64_t>(spins, 1) : (1ll << 23);
    const unsigned long long off = enable ? (1ull << 31) : 0ull;   // block counts stay below 2^31
    EFIE_CUDA(cudaMemcpyToSymbol(d_wait_spins, &lim, sizeof(lim)));
    EFIE_CUDA(cudaMemcpyToSymbol(d_wait_offset, &off, sizeof(off)));
    EFIE_CUDA(cudaDeviceSynchronize());
    return EFIE_OK;
}

efie_status efie_trsv_workspace(SolveWork &w) {
    int dev = 0, sms = 0, occ = 0;
    EFIE_CUDA(cudaGetDevice(&dev));
    EFIE_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    EFIE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_trsv<true>, 256, 0));
    int occ2 = 0;
    EFIE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ2, k_trsv<false>, 256, 0));
    occ = std::max(1, std::min(std::min(occ, occ2), 2));
    w.grid = std::max(1, std::min(w.nblk * w.B, occ * sms));
    const size_t bytes = sizeof(unsigned long long) * LINE * 2 * (size_t)w.B * w.grid;
    if (bytes > w.prog.bytes) {
        EFIE_TRY(w.prog.reserve(bytes));
        EFIE_CUDA(cudaMemset(w.prog.p, 0, bytes));  // epoch 0 < every real epoch
    }
    return EFIE_OK;
}

efie_status efie_trsv(efie_ctx *ctx, SolveWork &w, bool lower, const float2 *rhs, float2 *out, void *x, int epoch) {
    int grid = w.grid;
    const float *planes = w.planes.as<float>();
    const float2 *dinv = w.dinv.as<float2>();
    double2 *xd = static_cast<double2 *>(x);
    unsigned long long *prog = w.prog.as<unsigned long long>();
    char *ctl = w.ctl.as<char>();
    const int *active = w.active.as<int>();
    void *args[] = {(void *)&w.N,  (void *)&w.nblk, (void *)&w.B,    (void *)&planes, (void *)&w.pstride,
                    (void *)&w.ld, (void *)&dinv,   (void *)&w.dstride, (void *)&rhs, (void *)&out,
                    (void *)&w.vstride, (void *)&xd, (void *)&prog, (void *)&epoch, (void *)&ctl,
                    (void *)&active};
    const void *fn = lower ? (const void *)k_trsv<true> : (const void *)k_trsv<false>;
    EFIE_CUDA(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(256), args, 0, ctx->stream));
    return EFIE_OK;
}
