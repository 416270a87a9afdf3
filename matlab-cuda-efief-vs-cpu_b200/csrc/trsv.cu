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
// Nothing a CTA reads from the factors depends on a counter, so its tiles and
// diagonal inverses stream through a TMA ring ahead of the solve (k_trsv).
#include <algorithm>
#include <cstdint>


#include "efie_internal.h"
#include "solve.h"
#include "tma.h"

namespace {

using namespace efie_tma;

constexpr int NB = 64;
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

constexpr int TS = 3;                                          // stages of the tile ring
constexpr uint32_t STAGE_BYTES = 2u * NB * NB * sizeof(float);  // a 64 x 64 complex tile: 32 KB
constexpr uint32_t BOX_BYTES = 32u * 32u * sizeof(float);       // one 32 x 32 box of one plane
constexpr size_t TRSV_SMEM = TS * STAGE_BYTES + 1024 + 64;      // ring (1024-aligned) + barriers

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

// Columns quarter*16 .. +15 of row `row` of a staged tile: the tile is eight
// 32 x 32 boxes [plane][row half][column half] of 128-byte rows whose 16-byte
// chunk q sits at chunk q ^ (row mod 8) (the TMA 128B swizzle); a warp reads
// 32 consecutive rows, so each quarter-warp touches eight distinct chunks.
__device__ __forceinline__ void stage_row(float4 (&t)[8], const unsigned char *stage, int row, int quarter) {
    const int rh = row >> 5, lr = row & 31, ch = quarter >> 1, q0 = (quarter & 1) * 4;
#pragma unroll
    for (int pl = 0; pl < 2; pl++) {
        const unsigned char *box = stage + ((pl * 2 + rh) * 2 + ch) * BOX_BYTES + lr * 128;
#pragma unroll
        for (int c = 0; c < 4; c++)
            t[pl * 4 + c] = *reinterpret_cast<const float4 *>(box + (((q0 + c) ^ (lr & 7)) << 4));
    }
}

// Block-row solves of the items of one CTA.  Every 32 KB piece an item reads
// -- the 64 x 64 tiles of its block row (8 TMA boxes each) and then its
// diagonal inverse (one bulk copy) -- flows through a ring of TS stages fed
// by thread 0 in the CTA's item order, so the loads of later tiles, and of
// the next items, are in flight while the CTA waits for a solved block or
// works on the current one.  The right-hand side blocks y_jb are read from
// global memory after their publication (one block ahead when already
// published).
template <bool LOWER>
__global__ void __launch_bounds__(256, 2) k_trsv(const __grid_constant__ CUtensorMap map, int N, int nblk, int B,
                                                 const float2 *__restrict__ dinv, size_t dstride,
                                                 const float2 *__restrict__ rhsb, float2 *outb, int vstride,
                                                 double2 *__restrict__ xb, unsigned long long *prog, int epoch,
                                                 char *ctl, const int *__restrict__ active,
                                                 const int *__restrict__ fsrc) {
    extern __shared__ unsigned char dsm[];
    __shared__ float2 acc[NB];
    __shared__ float2 part[4][NB];
    __shared__ int avail_sh, ok, fail;
    unsigned char *ring = dsm + (((smem_u32(dsm) + 1023u) & ~1023u) - smem_u32(dsm));
    uint64_t *full = reinterpret_cast<uint64_t *>(ring + TS * STAGE_BYTES);
    const int tid = threadIdx.x;
    const int row = tid & 63, quarter = tid >> 6;
    const int G = gridDim.x;
    const unsigned long long tag = (unsigned long long)(unsigned)epoch << 32;
    const int dir = LOWER ? 0 : 1;
    const int items = nblk * B;
    auto live = [&](int it) -> bool {
        const int f = it % B;
        return active[f] && !*reinterpret_cast<const volatile int *>(ctl + 64 * f + 32);
    };
    // producer state (thread 0): the next piece is piece p_q of item p_it
    // (p_q < o: tile of block column q; p_q == o: the diagonal inverse)
    int p_it = blockIdx.x, p_q = 0, issued = 0;
    auto produce = [&]() {
        if (p_it >= items) return;
        const int o = p_it / B, b = LOWER ? o : nblk - 1 - o;
        const int f = fsrc ? fsrc[p_it - o * B] : p_it - o * B;   // the slot whose factors precondition it
        unsigned char *st = ring + (issued % TS) * STAGE_BYTES;
        uint64_t *bar = full + issued % TS;
        mbar_expect_tx(bar, STAGE_BYTES);
        if (p_q < o) {
            const int jb = LOWER ? p_q : nblk - 1 - p_q;
#pragma unroll
            for (int pl = 0; pl < 2; pl++)
#pragma unroll
                for (int rh = 0; rh < 2; rh++)
#pragma unroll
                    for (int ch = 0; ch < 2; ch++)
                        tma_load_4d(&map, st + ((pl * 2 + rh) * 2 + ch) * BOX_BYTES, jb * NB + ch * 32,
                                    b * NB + rh * 32, pl, f, bar);
        } else {
            bulk_g2s(st, dinv + dstride * f + (size_t)b * 2 * NB * NB + (LOWER ? 0 : NB * NB), STAGE_BYTES, bar);
        }
        issued++;
        if (++p_q > o) {
            p_q = 0;
            for (p_it += G; p_it < items && !live(p_it); p_it += G) {
            }
        }
    };
    if (tid == 0) {
        for (int s = 0; s < TS; s++) mbar_init(full + s, 1);
        mbar_init_fence();
        fail = 0;
        while (p_it < items && !live(p_it)) p_it += G;
        for (int s = 0; s < TS; s++) produce();
    }
    __syncthreads();
    int cc = 0;   // pieces consumed
    // wait for the next piece (every thread); the CTA decides together after its barrier
    auto take = [&]() -> const unsigned char * {
        if (!mbar_wait_bounded(full + cc % TS, (uint32_t)(cc / TS) & 1u)) fail = 1;
        return ring + (cc % TS) * STAGE_BYTES;
    };
    // thread 0 drains the pieces in flight before the CTA returns early
    auto drain = [&]() {
        if (tid != 0) return;
        for (int k = cc; k < issued; k++)
            if (!mbar_wait_bounded(full + k % TS, (uint32_t)(k / TS) & 1u)) return;
    };
    for (int it = blockIdx.x; it < items; it += G) {
        const int o = it / B, f = it - o * B;
        if (!live(it)) continue;
        const char *c = ctl + 64 * f;
        const volatile int *err = reinterpret_cast<const volatile int *>(c + 36);
        const int b = LOWER ? o : nblk - 1 - o;
        const float2 *rhs = rhsb + (size_t)vstride * f;
        float2 *out = outb + (size_t)vstride * f;
        unsigned long long *myctr = prog + ((size_t)(dir * B + f) * G + blockIdx.x) * LINE;
        const int r0 = b * NB;
        const int rows = min(NB, N - r0);
        if (tid < NB) acc[tid] = (tid < rows) ? rhs[r0 + tid] : make_float2(0.f, 0.f);
        if (tid == 0) ok = 1, avail_sh = 0;
        __syncthreads();
        // each thread keeps its quarter-row dot product in registers across the
        // dependencies; the CTA synchronises to wait for a block only when the
        // last observed count does not cover it (one count can cover many)
        float2 sdot = make_float2(0.f, 0.f);
        int avail = 0;
        float2 ynext[16];
        bool have_next = false;
        auto load_y = [&](float2 (&y)[16], int jb) {
            const float2 *ysrc = out + jb * NB + quarter * 16;
#pragma unroll
            for (int k = 0; k < 16; k++) y[k] = (jb * NB + quarter * 16 + k < N) ? ysrc[k] : make_float2(0.f, 0.f);
        };
        for (int q = 0; q < o; q++) {
            const int jb = LOWER ? q : nblk - 1 - q;
            if (q >= avail) {
                if (tid == 0) {
                    const unsigned long long v = wait_progress(myctr, tag | (unsigned long long)(q + 1), err);
                    if (!v) ok = 0;
                    avail_sh = (int)(v & 0xffffffffull);
                }
                __syncthreads();
                if (!ok) {
                    drain();
                    return;
                }
                avail = avail_sh;
            }
            // block jb of the solution: written by another CTA and published
            // before `avail` was read, then never changed in this launch
            float2 y16[16];
            if (have_next) {
#pragma unroll
                for (int k = 0; k < 16; k++) y16[k] = ynext[k];
            } else {
                load_y(y16, jb);
            }
            have_next = q + 1 < o && q + 1 < avail;
            if (have_next) load_y(ynext, LOWER ? jb + 1 : jb - 1);
            const unsigned char *st = take();
            if (!fail) {
                float4 t[8];
                stage_row(t, st, row, quarter);
                const float2 d = dot16(t, y16);
                sdot.x += d.x;
                sdot.y += d.y;
            }
            __syncthreads();
            if (fail) {
                if (tid == 0) atomicExch((int *)err, 2);
                drain();
                return;
            }
            if (tid == 0) produce();
            cc++;
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
        // y_b = inv(diagonal block) * acc; the inverse is row-major float2
        // [64][64] in the stage, read from column (k + row) mod 16 of the
        // thread's 16 so that a warp's 32 rows spread over the banks
        {
            const float2 *dst = reinterpret_cast<const float2 *>(take());
            float2 sv = make_float2(0.f, 0.f);
            if (!fail) {
                const float2 *drow = dst + row * NB + quarter * 16;
                const float2 *av = acc + quarter * 16;
                const int rot = row & 15;
#pragma unroll
                for (int k = 0; k < 16; k++) {
                    const int cix = (k + rot) & 15;
                    const float2 m = drow[cix], v = av[cix];
                    sv.x += m.x * v.x - m.y * v.y;
                    sv.y += m.x * v.y + m.y * v.x;
                }
            }
            part[quarter][row] = sv;
        }
        __syncthreads();
        if (fail) {
            if (tid == 0) atomicExch((int *)err, 2);
            drain();
            return;
        }
        if (tid == 0) produce();
        cc++;
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
    EFIE_CUDA(cudaFuncSetAttribute(k_trsv<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TRSV_SMEM));
    EFIE_CUDA(cudaFuncSetAttribute(k_trsv<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TRSV_SMEM));
    EFIE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_trsv<true>, 256, TRSV_SMEM));
    int occ2 = 0;
    EFIE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ2, k_trsv<false>, 256, TRSV_SMEM));
    occ = std::max(1, std::min(std::min(occ, occ2), 2));
    w.grid = std::max(1, std::min(w.nblk * w.B, occ * sms));
    const size_t bytes = sizeof(unsigned long long) * LINE * 2 * (size_t)w.B * w.grid;
    if (bytes > w.prog.bytes) {
        EFIE_TRY(w.prog.reserve(bytes));
        EFIE_CUDA(cudaMemset(w.prog.p, 0, bytes));  // epoch 0 < every real epoch
    }
    return EFIE_OK;
}

// The factors are read through the planes' tensor map (SolveWork::planes_map,
// encoded with the workspace): 32 x 32 boxes, zeros past row and column N.
efie_status efie_trsv(efie_ctx *ctx, SolveWork &w, bool lower, const float2 *rhs, float2 *out, void *x, int epoch) {
    int grid = w.grid;
    const float2 *dinv = w.dinv.as<float2>();
    double2 *xd = static_cast<double2 *>(x);
    unsigned long long *prog = w.prog.as<unsigned long long>();
    char *ctl = w.ctl.as<char>();
    const int *active = w.active.as<int>();
    const int *fsrc = w.fsrc_on ? w.fsrc.as<int>() : nullptr;
    void *args[] = {(void *)w.planes_map, (void *)&w.N,   (void *)&w.nblk,    (void *)&w.B,  (void *)&dinv,
                    (void *)&w.dstride,   (void *)&rhs,   (void *)&out,       (void *)&w.vstride,
                    (void *)&xd,          (void *)&prog,  (void *)&epoch,     (void *)&ctl,  (void *)&active,
                    (void *)&fsrc};
    const void *fn = lower ? (const void *)k_trsv<true> : (const void *)k_trsv<false>;
    EFIE_CUDA(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(256), args, TRSV_SMEM, ctx->stream));
    return EFIE_OK;
}
