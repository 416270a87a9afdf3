// Trailing-matrix update of the complex64 LU on the 5th-generation tensor
// cores: A22 -= L21 * U12.
//
// The complex product is realified into one real GEMM per 64-row block:
//     [ Re ]   [ Lr  -Li ]   [ Ur ]
//     [ Im ] = [ Li   Lr ] * [ Ui ]        (M' = 128 rows, K' = 2 kb)
// and every operand is split into two FP16 terms after an exact power-of-two
// scaling: each complex row of L21 by s_i and each column of U12 by t_j so
// that the largest magnitude of the row (column) over the update's K range
// lies in [1/2, 1); then x = hi + lo with hi = fp16(x), lo = fp16(x - hi)
// (22 significant bits, the precision of a TF32 pair at half the bytes).  The
// three products hi*hi + hi*lo + lo*hi accumulate in FP32 in tensor memory
// (TMEM, kind::f16, K = 16 per instruction) and the epilogue multiplies by
// 1/(s_i t_j), which is exact.  The update stays close to FP32 accuracy
// normwise (the LU is then refined in FP64).
//
// Operands are packed per LU step into 64B-swizzled K-major tiles (32 FP16
// per row) that sit contiguously in global memory, so each CTA fetches them
// with plain bulk copies (cp.async.bulk, the TMA engine; no multicast, local
// memory only).  One CTA computes two 128 x 256 accumulator tiles (2 x 64
// complex rows x 256 complex columns) in the 512 TMEM columns of its SM, both
// fed by the same B chunk, which halves the B bytes per MMA.  One elected
// thread issues tcgen05.mma over a 3-stage shared-memory ring of K' chunks --
// it issues chunk c's MMAs before waiting for chunk c-1's to retire, so the
// tensor pipe always holds queued work while the bulk loads run ahead.
// Meanwhile the other warps prefetch the CTA's rows of C into L2 (bulk
// prefetch), and at the end all eight warps drain TMEM with tcgen05.ld -- two
// warps per TMEM lane quarter, each taking half of the columns -- for the
// read-modify-write epilogue on the row-major planes, reading the next 32
// columns of C while they update the current ones.
// Every mbarrier wait is bounded; a timeout sets the device error flag.
#include <cstdint>

#include <cuda_fp16.h>

#include "solve.h"

namespace {

constexpr int KMAX = 256;        // largest complex K of one update (the outer LU block)
constexpr int TM = 128;          // accumulator rows (64 complex rows)
constexpr int TN = 256;          // accumulator columns (complex columns)
constexpr int KC = 32;           // fp16 elements per 64-byte swizzle row (one K' chunk)
constexpr int NCHUNK_MAX = 2 * KMAX / KC;   // K' = 2K -> up to 16 chunks
constexpr int A_TILE = TM * KC;       // halves per A tile (8 KB)
constexpr int B_TILE = TN * KC;       // halves per B tile (16 KB)
constexpr int MT = 2;            // 128-row accumulator tiles per CTA (TMEM columns: MT x 256)
constexpr int STAGE_HALVES = MT * 2 * A_TILE + 2 * B_TILE;   // hi/lo of MT A tiles and of B: 64 KB
constexpr int NSTAGE = 3;
constexpr int NBAR = 2 * NSTAGE + 1;  // full[NSTAGE], empty[NSTAGE], done
constexpr size_t GEMM_SMEM = sizeof(__half) * NSTAGE * STAGE_HALVES + 1024 + 8 * NBAR + 16 + sizeof(float) * TN;

// byte offset of element (row r, k) inside a K-major 64B-swizzled tile of
// fp16: the 16-byte chunk index (k / 8) XOR (r / 2) mod 4, 8-row atoms of 512 bytes
__host__ __device__ __forceinline__ uint32_t swz(uint32_t r, uint32_t k) {
    return r * 64u + ((((k >> 3) ^ (r >> 1)) & 3u) << 4) + ((k & 7u) << 1);
}

// 2^-e with max * 2^-e in [1/2, 1) (1 for a zero maximum)
__device__ __forceinline__ float pow2_scale(float mx) {
    if (!(mx > 0.f)) return 1.f;
    int e;
    frexpf(mx, &e);
    return ldexpf(1.f, -e);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Largest magnitude of a row of L over the 64-column blocks [b0, b1), and of a
// column of U over the 64-row blocks [b0, b1): the maxima are written with
// the factors (k_panels), so a scale costs at most four loads.
__device__ __forceinline__ float row_max(const float *lm, int row, int nblk, int b0, int b1) {
    float m = 0.f;
    for (int b = b0; b < b1; b++) m = fmaxf(m, lm[(size_t)row * nblk + b]);
    return m;
}
__device__ __forceinline__ float col_max(const float *um, int ld, int col, int b0, int b1) {
    float m = 0.f;
    for (int b = b0; b < b1; b++) m = fmaxf(m, um[(size_t)b * ld + col]);
    return m;
}

// ---------------------------------------------------------------------------
// Packing.  A: per 64-row block of L21 and K' chunk, a 128 x 32 tile (hi, lo).
// B: per 256-column block of U12 and K' chunk, a 256 x 32 tile (hi, lo).
// Tiles are built in shared memory in their final swizzled byte layout and
// written out with coalesced 16-byte stores.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void split_half(float v, __half &h, __half &l) {
    h = __float2half_rn(v);
    l = __float2half_rn(v - __half2float(h));
}

__global__ void __launch_bounds__(256) k_pack_a(int N, int r0, int r1, int kcol, int K, int nchunk,
                                                const float *__restrict__ planes, size_t pstride, int ld,
                                                const float *__restrict__ lmaxb, size_t mstride, int nblk,
                                                __half *__restrict__ outb, size_t ostride,
                                                const int *__restrict__ active) {
    __shared__ __align__(1024) __half hi[A_TILE];
    __shared__ __align__(1024) __half lo[A_TILE];
    __shared__ float rscale[64];
    const int f = blockIdx.z;
    if (!active[f]) return;
    const float *Ar = planes + pstride * f, *Ai = Ar + (size_t)ld * N;
    __half *out = outb + ostride * f;
    const int tile = blockIdx.x, chunk = blockIdx.y;
    if (threadIdx.x < 64) {
        const int row = r0 + tile * 64 + threadIdx.x;
        rscale[threadIdx.x] =
            row < r1 ? pow2_scale(row_max(lmaxb + mstride * f, row, nblk, kcol / 64, (kcol + K + 63) / 64)) : 0.f;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < A_TILE; e += 256) {
        const int r = e >> 5, kq = e & 31;           // consecutive threads: consecutive k
        const int kp = chunk * KC + kq;              // K' index
        const bool second = kp >= K;
        const int kk = second ? kp - K : kp;         // column within the L block
        const int rl = tile * 64 + (r & 63);         // complex row within the update
        const int row = r0 + rl;
        float v = 0.f;
        if (row < r1 && kk < K) {
            const size_t o = (size_t)row * ld + kcol + kk;
            if (r < 64) v = second ? -Ai[o] : Ar[o];     // [ Lr  -Li ]
            else v = second ? Ar[o] : Ai[o];            // [ Li   Lr ]
            v *= rscale[r & 63];                        // exact: a power of two
        }
        const uint32_t off = swz(r, kq) >> 1;
        split_half(v, hi[off], lo[off]);
    }
    __syncthreads();
    float4 *dst = reinterpret_cast<float4 *>(out + ((size_t)(tile * nchunk + chunk) * 2) * A_TILE);
    const float4 *h4 = reinterpret_cast<const float4 *>(hi), *l4 = reinterpret_cast<const float4 *>(lo);
    for (int e = threadIdx.x; e < A_TILE / 8; e += 256) {
        dst[e] = h4[e];
        dst[A_TILE / 8 + e] = l4[e];
    }
}

__global__ void __launch_bounds__(256) k_pack_b(int N, int c0, int c1, int krow, int K, int nchunk,
                                                const float *__restrict__ planes, size_t pstride, int ld,
                                                const float *__restrict__ umaxb, size_t mstride,
                                                __half *__restrict__ outb, size_t ostride,
                                                const int *__restrict__ active) {
    extern __shared__ __align__(1024) __half dynb[];
    __half *hi = dynb, *lo = dynb + B_TILE;
    __shared__ float cscale[TN];
    const int f = blockIdx.z;
    if (!active[f]) return;
    const float *Ar = planes + pstride * f, *Ai = Ar + (size_t)ld * N;
    __half *out = outb + ostride * f;
    const int tile = blockIdx.x, chunk = blockIdx.y;
    {
        const int col = c0 + tile * TN + threadIdx.x;   // 256 threads: one column each
        cscale[threadIdx.x] =
            col < c1 ? pow2_scale(col_max(umaxb + mstride * f, ld, col, krow / 64, (krow + K + 63) / 64)) : 0.f;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < B_TILE; e += 256) {
        const int kq = e >> 8, n = e & 255;          // consecutive threads: consecutive columns
        const int kp = chunk * KC + kq;
        const bool second = kp >= K;
        const int kk = second ? kp - K : kp;
        const int cl = tile * TN + n;
        const int col = c0 + cl;
        float v = 0.f;
        if (col < c1 && kk < K) {
            const size_t o = (size_t)(krow + kk) * ld + col;
            v = (second ? Ai[o] : Ar[o]) * cscale[n];   // [ Ur ; Ui ], exact scaling
        }
        const uint32_t off = swz(n, kq) >> 1;
        split_half(v, hi[off], lo[off]);
    }
    __syncthreads();
    float4 *dst = reinterpret_cast<float4 *>(out + ((size_t)(tile * nchunk + chunk) * 2) * B_TILE);
    const float4 *h4 = reinterpret_cast<const float4 *>(hi), *l4 = reinterpret_cast<const float4 *>(lo);
    for (int e = threadIdx.x; e < B_TILE / 8; e += 256) {
        dst[e] = h4[e];
        dst[B_TILE / 8 + e] = l4[e];
    }
}

// ---------------------------------------------------------------------------
// tcgen05 / mbarrier / bulk-copy primitives (inline PTX)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: false (and the error flag set) after ~1 s of polling.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *err) {
    for (long long i = 0; i < (1ll << 22); i++) {
        if (mbar_try_wait(bar, parity)) return true;
        if (i > 64) __nanosleep(64);
    }
    atomicExch(err, 3);
    return false;
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ uint64_t desc_sw64(const void *smem_tile) {
    const uint32_t a = smem_u32(smem_tile);
    uint64_t d = 0;
    d |= (uint64_t)((a & 0x3FFFFu) >> 4);      // start address
    d |= (uint64_t)1 << 16;                    // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(512 >> 4) << 32;           // stride byte offset: 8 rows x 64 B
    d |= (uint64_t)1 << 46;                    // descriptor version (sm_100)
    d |= (uint64_t)4 << 61;                    // SWIZZLE_64B
    return d;
}

// kind::f16, D = F32, A = B = F16, both K-major, N = 256, M = 128
constexpr uint32_t IDESC = (1u << 4) | (0u << 7) | (0u << 10) | ((uint32_t)(TN >> 3) << 17) |
                           ((uint32_t)(TM >> 4) << 24);

__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(IDESC), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// ---------------------------------------------------------------------------
// The update kernel: grid (ceil(m/256), ceil(m/64)), 128 threads.
// ---------------------------------------------------------------------------
// C[r0:r1, c0:c1] -= (packed A) * (packed B) for the CTA's tiles; grid
// (column tiles, pairs of 64-row tiles, frequency), 256 threads.
__global__ void __launch_bounds__(256, 1) k_update_tc(int N, int r0, int r1, int c0, int c1, int nchunk, int mt,
                                                      const __half *__restrict__ Apackb, size_t astride,
                                                      const __half *__restrict__ Bpackb, size_t bstride,
                                                      const float *__restrict__ lmaxb, const float *__restrict__ umaxb,
                                                      size_t mstride, int nblk, int kcol, int krow, int K,
                                                      float *__restrict__ planes, size_t pstride, int ld,
                                                      char *__restrict__ ctl, const int *__restrict__ active) {
    const int f = blockIdx.z;
    if (!active[f]) return;
    const __half *Apack = Apackb + astride * f, *Bpack = Bpackb + bstride * f;
    const float *lm = lmaxb + mstride * f, *um = umaxb + mstride * f;
    float *Ar = planes + pstride * f, *Ai = Ar + (size_t)ld * N;
    int *err = reinterpret_cast<int *>(ctl + 64 * f + 36);
    extern __shared__ uint8_t dyn_raw[];
    // 1024-byte alignment for the swizzled tiles
    __half *stage = reinterpret_cast<__half *>((reinterpret_cast<uintptr_t>(dyn_raw) + 1023) & ~(uintptr_t)1023);
    uint64_t *bars = reinterpret_cast<uint64_t *>(stage + NSTAGE * STAGE_HALVES);  // full[], empty[], done
    uint64_t *full = bars, *empty = bars + NSTAGE, *done = bars + 2 * NSTAGE;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + NBAR);
    int *ok_sh = reinterpret_cast<int *>(tmem_slot + 1);
    float *col_is = reinterpret_cast<float *>(bars + 8);   // 16-byte aligned: inverse column scales of the tile
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tile_n = blockIdx.x, tile_m0 = blockIdx.y * MT;
    const int nm = min(MT, mt - tile_m0);            // accumulator tiles of this CTA (1 or 2)

    if (tid == 0) {
        for (int i = 0; i < NBAR; i++) mbar_init(&bars[i], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(MT * TN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    bool ok = true;
    if (tid == 0) *ok_sh = 1;
    if (tid == 0) {
        const __half *gb = Bpack + (size_t)tile_n * nchunk * 2 * B_TILE;
        const uint32_t abytes = sizeof(__half) * 2 * A_TILE, bbytes = sizeof(__half) * 2 * B_TILE;
        auto load = [&](int c) {
            __half *st = stage + (c % NSTAGE) * STAGE_HALVES;
            mbar_expect_tx(&full[c % NSTAGE], nm * abytes + bbytes);
            for (int mi = 0; mi < nm; mi++)
                bulk_g2s(st + mi * 2 * A_TILE, Apack + ((size_t)(tile_m0 + mi) * nchunk + c) * 2 * A_TILE, abytes,
                         &full[c % NSTAGE]);
            bulk_g2s(st + MT * 2 * A_TILE, gb + (size_t)c * 2 * B_TILE, bbytes, &full[c % NSTAGE]);
        };
        for (int c = 0; c < NSTAGE && c < nchunk; c++) load(c);
        for (int c = 0; c < nchunk && ok; c++) {
            const int sidx = c % NSTAGE;
            if (!mbar_wait(&full[sidx], (c / NSTAGE) & 1, err)) { ok = false; break; }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const __half *st = stage + sidx * STAGE_HALVES;
            const uint64_t bhi = desc_sw64(st + MT * 2 * A_TILE), blo = desc_sw64(st + MT * 2 * A_TILE + B_TILE);
            for (int mi = 0; mi < nm; mi++) {
                const uint64_t ahi = desc_sw64(st + mi * 2 * A_TILE), alo = desc_sw64(st + mi * 2 * A_TILE + A_TILE);
                const uint32_t acc = tmem + (uint32_t)(mi * TN);
#pragma unroll
                for (int kk = 0; kk < KC / 16; kk++) {
                    const uint64_t adv = (uint64_t)((kk * 32) >> 4);   // 16 fp16 = 32 bytes along K
                    // small terms first, then the leading product
                    mma_f16(acc, alo + adv, bhi + adv, (c > 0 || kk > 0) ? 1u : 0u);
                    mma_f16(acc, ahi + adv, blo + adv, 1u);
                    mma_f16(acc, ahi + adv, bhi + adv, 1u);
                }
            }
            mma_commit(&empty[sidx]);   // stage sidx free once these MMAs have read it
            // refill the stage of chunk c - 1: its MMAs were queued ahead of chunk
            // c's, so waiting for them leaves chunk c's MMAs on the tensor pipe
            const int cp = c - 1;
            if (cp >= 0 && cp + NSTAGE < nchunk) {
                if (!mbar_wait(&empty[cp % NSTAGE], (cp / NSTAGE) & 1, err)) { ok = false; break; }
                load(cp + NSTAGE);
            }
        }
        mma_commit(done);                  // all MMAs of this CTA done
        if (!ok) *ok_sh = 0;
    } else if (warp > 0) {
        // inverse column scales of the tile into shared memory
        for (int j = tid - 32; j < TN; j += 224) {
            const int col = c0 + tile_n * TN + j;
            col_is[j] = (col < c1) ? 1.f / pow2_scale(col_max(um, ld, col, krow / 64, (krow + K + 63) / 64)) : 0.f;
        }
        // C rows of this CTA into L2 while the MMAs run: (accumulator, plane, row) segments
        const int ncol = min(TN, c1 - (c0 + tile_n * TN));
        const uint32_t bytes = (uint32_t)((ncol * 4 + 15) & ~15);
        for (int e = tid - 32; e < nm * 2 * 64; e += 224) {
            const int mi = e >> 7, pl = (e >> 6) & 1, rr = e & 63;
            const int row = r0 + (tile_m0 + mi) * 64 + rr;
            if (row < r1 && ncol > 0) {
                const float *src = (pl ? Ai : Ar) + (size_t)row * ld + c0 + tile_n * TN;
                asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
            }
        }
    }
    __syncthreads();
    // every thread waits for the accumulators (bounded); the decision is made
    // uniform per warp because tcgen05.ld is a warp-collective instruction
    bool have = mbar_wait(done, 0, err);
    have = __all_sync(0xffffffffu, have) && (*ok_sh != 0);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (have) {
        // TMEM lane quarter of this warp (tcgen05.ld reaches lanes 32 (warp mod 4) ...)
        const int quarter = warp & 3;
        const int half = quarter & 1;               // rows 0-31 or 32-63 of a complex block
        float *plane = (quarter < 2) ? Ar : Ai;     // quarters 0,1: real part; 2,3: imaginary part
        constexpr int NJ = TN / 32;
        const int j0 = (warp >> 2) * (NJ / 2), j1 = j0 + NJ / 2;   // this warp's half of the columns
        for (int mi = 0; mi < nm; mi++) {
            const int rl = (tile_m0 + mi) * 64 + half * 32 + lane;   // complex row within the update
            const int row = r0 + rl;
            const bool rok = row < r1;
            const float rs = rok ? 1.f / pow2_scale(row_max(lm, row, nblk, kcol / 64, (kcol + K + 63) / 64)) : 0.f;
            const uint32_t tbase = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(mi * TN);
            float *prow = plane + (size_t)(rok ? row : r0) * ld + c0 + tile_n * TN;
            const int ncol = c1 - (c0 + tile_n * TN);   // valid columns of this tile (may exceed TN)
            // C of chunk j + 1 is read while chunk j is updated
            float4 cur[8], nxt[8];
            auto fetch = [&](int j, float4 (&d)[8]) {
                if (rok && (j + 1) * 32 <= ncol) {
                    const float4 *p4 = reinterpret_cast<const float4 *>(prow + j * 32);
#pragma unroll
                    for (int q = 0; q < 8; q++) d[q] = p4[q];
                }
            };
            fetch(j0, cur);
#pragma unroll 1
            for (int j = j0; j < j1; j++) {
                if (j + 1 < j1) fetch(j + 1, nxt);
                uint32_t v[32];
                tmem_ld32(tbase + j * 32, v);
                const int col0 = j * 32;
                if (rok && col0 < ncol) {
                    float *p = prow + col0;
                    if (col0 + 32 <= ncol) {
                        float4 *p4 = reinterpret_cast<float4 *>(p);
#pragma unroll
                        for (int q = 0; q < 8; q++) {
                            const float4 cs = *reinterpret_cast<const float4 *>(col_is + col0 + 4 * q);
                            float4 a = cur[q];
                            a.x -= __uint_as_float(v[4 * q]) * (rs * cs.x);
                            a.y -= __uint_as_float(v[4 * q + 1]) * (rs * cs.y);
                            a.z -= __uint_as_float(v[4 * q + 2]) * (rs * cs.z);
                            a.w -= __uint_as_float(v[4 * q + 3]) * (rs * cs.w);
                            p4[q] = a;
                        }
                    } else {
#pragma unroll
                        for (int q = 0; q < 32; q++)
                            if (col0 + q < ncol) p[q] -= __uint_as_float(v[q]) * (rs * col_is[col0 + q]);
                    }
                }
#pragma unroll
                for (int q = 0; q < 8; q++) cur[q] = nxt[q];
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(MT * TN));
    }
}

}  // namespace

static bool g_tc_disabled = false;

efie_status efie_tc_attrs() {
    static bool done = false;
    if (done) return EFIE_OK;
    EFIE_CUDA(cudaFuncSetAttribute(k_update_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GEMM_SMEM));
    EFIE_CUDA(cudaFuncSetAttribute(k_pack_b, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)(sizeof(__half) * 2 * B_TILE)));
    done = true;
    return EFIE_OK;
}

extern "C" void efie_debug_disable_tensor_cores(int disable) { g_tc_disabled = disable != 0; }

// Staging for the largest update of an N x N LU (per frequency slot), and the
// kernel attributes: done when the workspace is created, so that the factor
// sequence allocates nothing and can be captured into a CUDA graph.
efie_status efie_gemm_workspace(SolveWork &w) {
    EFIE_TRY(efie_tc_attrs());
    const int mt0 = (w.N + 63) / 64, nt0 = (w.N + TN - 1) / TN;
    const size_t astride = (size_t)mt0 * NCHUNK_MAX * 2 * A_TILE, bstride = (size_t)nt0 * NCHUNK_MAX * 2 * B_TILE;
    EFIE_TRY(w.packA.reserve(sizeof(__half) * astride * w.B));
    EFIE_TRY(w.packB.reserve(sizeof(__half) * bstride * w.B));
    EFIE_TRY(w.packA2.reserve(sizeof(__half) * astride * w.B));
    EFIE_TRY(w.packB2.reserve(sizeof(__half) * bstride * w.B));
    return EFIE_OK;
}

// C[r0:r1, c0:c1] -= L[r0:r1, kcol:kcol+K] * U[krow:krow+K, c0:c1] for every
// active frequency: tensor cores when the block spans enough work, CUDA cores
// otherwise.
efie_status efie_gemm_update(efie_ctx *ctx, SolveWork &w, int r0, int r1, int c0, int c1, int kcol, int krow, int K,
                             int nact, int slot) {
    const int rows = r1 - r0, cols = c1 - c0;
    if (rows <= 0 || cols <= 0 || K <= 0) return EFIE_OK;
    const bool tc = !g_tc_disabled && K <= KMAX && (double)rows * cols >= 64.0 * 256.0 && cols >= 96;
    if (!tc) {
        for (int k0 = 0; k0 < K; k0 += 64)
            EFIE_TRY(efie_update_simt(ctx, w, r0, r1, c0, c1, kcol + k0, krow + k0, std::min(64, K - k0), nact));
        return EFIE_OK;
    }
    EFIE_TRY(efie_tc_attrs());
    const int N = w.N, B = w.B;
    cudaStream_t st = ctx->stream;
    const int mt = (rows + 63) / 64, nt = (cols + TN - 1) / TN;
    const int nchunk = (2 * K + KC - 1) / KC;
    // per-frequency staging sized for the largest update of an N x N LU
    const int mt0 = (N + 63) / 64, nt0 = (N + TN - 1) / TN;
    const size_t astride = (size_t)mt0 * NCHUNK_MAX * 2 * A_TILE, bstride = (size_t)nt0 * NCHUNK_MAX * 2 * B_TILE;
    DevBuf &pA = slot ? w.packA2 : w.packA, &pB = slot ? w.packB2 : w.packB;
    EFIE_TRY(pA.reserve(sizeof(__half) * astride * B));
    EFIE_TRY(pB.reserve(sizeof(__half) * bstride * B));
    float *planes = w.planes.as<float>();
    const int *active = w.active.as<int>();
    const float *lmax = w.lmax.as<float>(), *umax = w.umax.as<float>();
    KernelLog &log = ctx->log;
    size_t tok = log.begin(st);
    k_pack_a<<<dim3(mt, nchunk, B), 256, 0, st>>>(N, r0, r1, kcol, K, nchunk, planes, w.pstride, w.ld, lmax,
                                                  w.mstride, w.nblk, pA.as<__half>(), astride, active);
    k_pack_b<<<dim3(nt, nchunk, B), 256, sizeof(__half) * 2 * B_TILE, st>>>(
        N, c0, c1, krow, K, nchunk, planes, w.pstride, w.ld, umax, w.mstride, pB.as<__half>(), bstride, active);
    EFIE_CUDA(cudaGetLastError());
    log.end(EFIE_K_PANEL, st, tok, 0.0, 2);
    tok = log.begin(st);
    k_update_tc<<<dim3(nt, (mt + MT - 1) / MT, B), 256, GEMM_SMEM, st>>>(
        N, r0, r1, c0, c1, nchunk, mt, pA.as<__half>(), astride, pB.as<__half>(), bstride, lmax, umax, w.mstride,
        w.nblk, kcol, krow, K, planes, w.pstride, w.ld, w.ctl.as<char>(), active);
    EFIE_CUDA(cudaGetLastError());
    log.end(EFIE_K_GEMM, st, tok, 8.0 * (double)rows * cols * K * nact);
    return EFIE_OK;
}
