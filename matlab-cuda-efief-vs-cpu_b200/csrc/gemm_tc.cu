// Trailing-matrix update of the complex64 LU on the 5th-generation tensor
// cores: A22 -= L21 * U12.
//
// The complex product is written as four real products on separate real and
// imaginary tiles,
//     Re += Lr Ur - Li Ui        Im += Lr Ui + Li Ur,
// with the minus sign taken by the MMA's negate-A bit, so no operand is
// duplicated.  Every operand is split into two FP16 terms after an exact
// power-of-two scaling: each complex row of L21 by s_i and each column of
// U12 by t_j so that the largest magnitude of the row (column) over the
// update's K range lies in [2^14, 2^15); then x = hi + lo with hi = fp16(x),
// lo = fp16(x - hi) (22 significant bits, the lo half a normal FP16 number
// for entries down to 2^-18 of the maximum).  The three products hi*hi + hi*lo
// + lo*hi accumulate in FP32 in tensor memory (TMEM, kind::f16, K = 16 per
// instruction) and the epilogue multiplies by 1/(s_i t_j), which is exact.
// The update stays close to FP32 accuracy normwise (the LU is then refined in
// FP64).
//
// Operands are packed once per panel (the panel kernel packs the 64-wide
// blocks of the panel chain itself) into planes of 64B-swizzled K-major rows
// (32 FP16 per row) in which any 128 rows are contiguous, so each CTA fetches
// a K chunk of its operands with eight plain bulk copies (cp.async.bulk, the
// TMA engine; local memory only) from any row offset of the panel.  Two CTAs on the two SMs of a TPC form a
// cluster and compute one 256 x 256 complex tile with cta_group::2 MMAs
// (M = 256): each SM holds 128 rows of L21 (real and imaginary, hi and lo)
// and half of the tile's 256 columns of U12, and keeps the real and the
// imaginary accumulator of its 128 rows x 256 columns in its 512 TMEM
// columns.  Per MMA cycle an SM thus reads half the operand bytes of a
// realified single-SM tile.  One thread of the even CTA issues the MMAs over
// a 3-stage ring of K chunks (chunk c's MMAs are queued before the stage of
// chunk c-1 is refilled); the odd CTA's producer forwards the arrival of its
// half of each chunk to the even CTA's barrier, and the MMA completions are
// committed to the barriers of both CTAs.  Meanwhile the other warps prefetch
// the CTA's rows of C into L2 (bulk prefetch).  At the end all eight warps
// drain TMEM with tcgen05.ld -- four lane quarters x {real, imaginary} --,
// scale and negate each 32 x 32 block into a 128B-swizzled shared-memory tile
// and hand it to a bulk tensor reduction (cp.reduce.async.bulk.tensor .add),
// so the read-modify-write of C happens in L2 and the SM never loads C; the
// reductions drain while the next CTA on the SM runs its MMAs.  Each element
// of C receives exactly one addition per update (deterministic); rows and
// columns of a tile past the update's edge add exact zeros.
// Every mbarrier wait is bounded; a timeout sets the device error flag.
#include <cstdint>

#include <cuda.h>
#include <cuda_fp16.h>
#include <cudaTypedefs.h>

#include "solve.h"
#include "tma.h"

namespace {

constexpr int KMAX = 512;        // largest complex K of one update (the outer LU block)
constexpr int TR = 128;          // complex rows of L21 per CTA (one TMEM lane each)
constexpr int TM = 2 * TR;       // complex rows of the pair's tile (MMA M)
constexpr int KC = 32;           // fp16 elements per 64-byte swizzle row (one K chunk)
constexpr int NCHUNK_MAX = KMAX / KC;
constexpr int SUB = TR * KC;     // halves per 128 x 32 sub-tile (8 KB)
// a packed K chunk of one 128-row (128-column) tile: re hi, re lo, im hi, im lo
constexpr int CHUNK_HALVES = 4 * SUB;                      // 32 KB

// Tile shapes of the pair: TM x BN complex entries, BN = 256 or 128 columns.
// Each CTA holds TR rows of L and BN/2 columns of U per K chunk; the real and
// imaginary accumulators take 2 BN TMEM columns.  BN = 128 halves the U bytes
// and the drain per tile, so a 4-stage ring fits and narrow updates (the
// panel chain's last blocks) waste fewer columns.
template <int BN>
struct Tile {
    static constexpr int UH = BN / 2;                           // U columns per CTA
    static constexpr int USUB = UH * KC;                        // halves per U component sub-tile
    static constexpr int STAGE = CHUNK_HALVES + 4 * USUB;       // L chunk + U half chunk
    // stages of the ring: 192 KB for BN = 256 (one CTA per SM); 96 KB for
    // BN = 128, so that two CTAs (pairs) share an SM and one's set-up, drain
    // and reductions overlap the other's MMAs (2 x 256 TMEM columns)
    static constexpr int NST = BN == 256 ? 3 : 2;
    static constexpr int CTAS = BN == 256 ? 1 : 2;              // CTAs per SM
    // 4 KB reduction tiles per epilogue warp in the freed stages (at most 4)
    static constexpr int ER = (int)(NST * STAGE * sizeof(__half) / (8 * 4096)) < 4
                                  ? (int)(NST * STAGE * sizeof(__half) / (8 * 4096))
                                  : 4;
    static constexpr int NBAR = 3 * NST + 1;                    // full[], empty[], pair_full[], done
    static constexpr int BAR_WORDS = (NBAR + 1 + 1) & ~1;       // + TMEM slot and flag, 16-byte aligned
    static constexpr size_t SMEM = sizeof(__half) * NST * STAGE + 1024 + 8 * BAR_WORDS + sizeof(float) * BN;
};

__host__ __device__ __forceinline__ uint32_t swz(uint32_t r, uint32_t k) { return efie_swz64(r, k); }
__device__ __forceinline__ float pow2_scale(float mx) { return efie_pow2_scale(mx); }

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
// Packing: a CTA builds the four components (re hi, re lo, im hi, im lo) of
// 128 rows of L21 (columns of U12) and one K chunk in shared memory, in their
// swizzled byte layout, and writes each as one contiguous 8 KB block of its
// plane.  Rows (columns) past the panel's edge are zero.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void split_half(float v, __half &h, __half &l) {
    h = __float2half_rn(v);
    l = __float2half_rn(v - __half2float(h));
}

// four consecutive values times the scale, split into hi and lo halves, each
// set of four stored as one 8-byte word (4 consecutive k of a swizzled row)
__device__ __forceinline__ void split4(const float4 &v, float sc, __half *hi, __half *lo) {
    __half h[4], l[4];
    split_half(v.x * sc, h[0], l[0]);
    split_half(v.y * sc, h[1], l[1]);
    split_half(v.z * sc, h[2], l[2]);
    split_half(v.w * sc, h[3], l[3]);
    *reinterpret_cast<uint2 *>(hi) = *reinterpret_cast<const uint2 *>(h);
    *reinterpret_cast<uint2 *>(lo) = *reinterpret_cast<const uint2 *>(l);
}

// the four 128-row component tiles of one chunk to their planes
__device__ __forceinline__ void store_planes(const __half *t, __half *dst, int pitch) {
    for (int e = threadIdx.x; e < CHUNK_HALVES / 8; e += blockDim.x) {
        const int comp = e / (SUB / 8), i = e % (SUB / 8);
        reinterpret_cast<float4 *>(dst + (size_t)comp * pitch * KC)[i] = reinterpret_cast<const float4 *>(t)[e];
    }
}

__global__ void __launch_bounds__(256) k_pack_l(int N, int r0, int r1, int kcol, int K, int pitch,
                                                const float *__restrict__ planes, size_t pstride, int ld,
                                                const float *__restrict__ lmaxb, size_t mstride, int nblk,
                                                __half *__restrict__ outb, size_t ostride,
                                                const int *__restrict__ active) {
    __shared__ __align__(1024) __half t[CHUNK_HALVES];
    __shared__ float rscale[TR];
    const int f = blockIdx.z;
    if (!active[f]) return;
    const float *Ar = planes + pstride * f, *Ai = Ar + (size_t)ld * N;
    const int tile = blockIdx.x, chunk = blockIdx.y;
    if (threadIdx.x < TR) {
        const int row = r0 + tile * TR + threadIdx.x;
        rscale[threadIdx.x] =
            row < r1 ? pow2_scale(row_max(lmaxb + mstride * f, row, nblk, kcol / 64, (kcol + K + 63) / 64)) : 0.f;
    }
    __syncthreads();
    // four groups of four consecutive k per thread (eight 16-byte loads in
    // flight), split into halves that sit next to each other in the swizzled
    // row: one 8-byte store per component and group
    float4 vr[4], vi[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int e = threadIdx.x + 256 * i;
        const int r = e >> 3, kq = (e & 7) * 4;
        const int k = chunk * KC + kq;
        const int row = r0 + tile * TR + r;
        vr[i] = vi[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (row < r1) {
            const size_t o = (size_t)row * ld + kcol + k;
            if (k + 3 < K) {
                vr[i] = __ldg(reinterpret_cast<const float4 *>(Ar + o));
                vi[i] = __ldg(reinterpret_cast<const float4 *>(Ai + o));
            } else {
                float *pr = &vr[i].x, *pi = &vi[i].x;
                for (int j = 0; j < 4 && k + j < K; j++) pr[j] = Ar[o + j], pi[j] = Ai[o + j];
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int e = threadIdx.x + 256 * i;
        const int r = e >> 3, kq = (e & 7) * 4;
        const float sc = rscale[r];                   // exact: a power of two
        const uint32_t off = swz(r, kq) >> 1;
        split4(vr[i], sc, t + off, t + SUB + off);
        split4(vi[i], sc, t + 2 * SUB + off, t + 3 * SUB + off);
    }
    __syncthreads();
    store_planes(t, outb + ostride * f + ((size_t)chunk * 4 * pitch + (size_t)tile * TR) * KC, pitch);
}

__global__ void __launch_bounds__(256) k_pack_u(int N, int c0, int c1, int krow, int K, int pitch,
                                                const float *__restrict__ planes, size_t pstride, int ld,
                                                const float *__restrict__ umaxb, size_t mstride,
                                                __half *__restrict__ outb, size_t ostride,
                                                const int *__restrict__ active) {
    __shared__ __align__(1024) __half t[CHUNK_HALVES];
    __shared__ float cscale[TR];
    const int f = blockIdx.z;
    if (!active[f]) return;
    const float *Ar = planes + pstride * f, *Ai = Ar + (size_t)ld * N;
    const int tile = blockIdx.x, chunk = blockIdx.y;
    if (threadIdx.x < TR) {
        const int col = c0 + tile * TR + threadIdx.x;
        cscale[threadIdx.x] =
            col < c1 ? pow2_scale(col_max(umaxb + mstride * f, ld, col, krow / 64, (krow + K + 63) / 64)) : 0.f;
    }
    __syncthreads();
    // one column and four consecutive k per thread and group (loads coalesced
    // across the warp's consecutive columns), four groups in flight
    float4 vr[4], vi[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int e = threadIdx.x + 256 * i;
        const int n = e & (TR - 1), kq = (e >> 7) * 4;
        const int k = chunk * KC + kq;
        const int col = c0 + tile * TR + n;
        float *pr = &vr[i].x, *pi = &vi[i].x;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            pr[j] = pi[j] = 0.f;
            if (col < c1 && k + j < K) {
                const size_t o = (size_t)(krow + k + j) * ld + col;
                pr[j] = Ar[o];
                pi[j] = Ai[o];
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int e = threadIdx.x + 256 * i;
        const int n = e & (TR - 1), kq = (e >> 7) * 4;
        const float sc = cscale[n];
        const uint32_t off = swz(n, kq) >> 1;
        split4(vr[i], sc, t + off, t + SUB + off);
        split4(vi[i], sc, t + 2 * SUB + off, t + 3 * SUB + off);
    }
    __syncthreads();
    store_planes(t, outb + ostride * f + ((size_t)chunk * 4 * pitch + (size_t)tile * TR) * KC, pitch);
}

// ---------------------------------------------------------------------------
// tcgen05 / mbarrier / bulk-copy / cluster primitives (inline PTX)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// try_wait with acquire at cluster scope: also orders what the peer CTA
// released before its remote arrive
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
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

// address of the same shared-memory object in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t peer_addr(const void *p, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
    return r;
}

__device__ __forceinline__ void mbar_arrive_remote(uint32_t cluster_addr) {
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr) : "memory");
}

__device__ __forceinline__ void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// C[f][plane][y .. y+31][x .. x+31] += the 32 x 32 fp32 tile at `src`
// (128B-swizzled rows); coordinates past the tensor's edge are skipped
__device__ __forceinline__ void reduce_add_tile(const CUtensorMap *map, const float *src, int x, int y, int plane,
                                                int f) {
    asm volatile(
        "cp.reduce.async.bulk.tensor.4d.global.shared::cta.add.bulk_group [%0, {%2, %3, %4, %5}], [%1];" ::"l"(
            reinterpret_cast<uint64_t>(map)),
        "r"(smem_u32(src)), "r"(x), "r"(y), "r"(plane), "r"(f)
        : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

template <int N>
__device__ __forceinline__ void bulk_wait_read() {
    asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
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

// kind::f16, D = F32, A = B = F16, both K-major, M = 256 (CTA pair), N = 256;
// bit 13 negates A
template <int BN>
struct Idesc {
    static constexpr uint32_t POS = (1u << 4) | (0u << 7) | (0u << 10) | ((uint32_t)(BN >> 3) << 17) |
                                    ((uint32_t)(TM >> 4) << 24);
    static constexpr uint32_t NEG_A = POS | (1u << 13);
};

__device__ __forceinline__ void mma_pair(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

// arrive on the barrier at a shared::cluster address (this CTA's or the peer's)
// once every MMA issued so far by this thread has completed
__device__ __forceinline__ void mma_commit(uint32_t cluster_bar) {
    asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(cluster_bar)
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

// Column tiles (width bn) of row pair p in the lower-triangle mode: those
// whose first column block of width kb does not lie right of the pair's last
// row block.
__host__ __device__ __forceinline__ int tri_cols(int p, int nct, int kb, int bn) {
    const int qr = (p * TM + TM - 1) / kb;
    const int n = ((qr + 1) * kb + bn - 1) / bn;
    return n < nct ? n : nct;
}

// ---------------------------------------------------------------------------
// The update kernel.  C[r0:r1, c0:c1] -= (packed L) * (packed U) for the
// pair's 256 x BN tile; grid (2 x column tiles, row-pair tiles, frequency),
// clusters of two CTAs along x, 256 threads.
// ---------------------------------------------------------------------------
template <int BN>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(256, Tile<BN>::CTAS)
    k_update_tc(const __grid_constant__ CUtensorMap cmap, int N, int r0, int r1, int c0, int c1, int nchunk,
                const __half *__restrict__ Lpackb, size_t lstride, int lpitch, int loff,
                const __half *__restrict__ Upackb, size_t ustride, int upitch, int uoff, const float *__restrict__ lmaxb,
                const float *__restrict__ umaxb, size_t mstride, int nblk, int kcol, int krow, int K,
                float *__restrict__ planes, size_t pstride, int ld, char *__restrict__ ctl,
                const int *__restrict__ active, int tri_kb) {
    const int f = blockIdx.z;
    if (!active[f]) return;   // both CTAs of a cluster share f
    using T = Tile<BN>;
    constexpr int NSTAGE = T::NST;
    int ct = blockIdx.x >> 1;   // BN-column tile of the pair
    int rp = blockIdx.y;        // 256-row tile of the pair
    if (tri_kb > 0) {
        // lower tiles of a square block in row order (both CTAs of the pair
        // map the same x to the same tile)
        const int npr = (r1 - r0 + TM - 1) / TM, nct = (c1 - c0 + BN - 1) / BN;
        rp = 0;
        while (rp < npr - 1) {
            const int nc = tri_cols(rp, nct, tri_kb, BN);
            if (ct < nc) break;
            ct -= nc;
            rp++;
        }
        if (ct >= tri_cols(rp, nct, tri_kb, BN)) return;
    }
    const uint32_t rank = cluster_rank();
    const bool leader = rank == 0;
    const __half *Lpack = Lpackb + lstride * f, *Upack = Upackb + ustride * f;
    const float *lm = lmaxb + mstride * f, *um = umaxb + mstride * f;
    float *Ar = planes + pstride * f, *Ai = Ar + (size_t)ld * N;
    int *err = reinterpret_cast<int *>(ctl + 64 * f + 36);
    extern __shared__ uint8_t dyn_raw[];
    // 1024-byte alignment for the swizzled tiles (the same offset in both CTAs)
    __half *stage = reinterpret_cast<__half *>((reinterpret_cast<uintptr_t>(dyn_raw) + 1023) & ~(uintptr_t)1023);
    uint64_t *bars = reinterpret_cast<uint64_t *>(stage + NSTAGE * T::STAGE);
    uint64_t *full = bars, *empty = bars + NSTAGE, *pfull = bars + 2 * NSTAGE, *done = bars + 3 * NSTAGE;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + T::NBAR);
    int *ok_sh = reinterpret_cast<int *>(tmem_slot + 1);
    float *col_is = reinterpret_cast<float *>(bars + T::BAR_WORDS);   // 16-byte aligned: inverse column scales
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int rtile = rp * 2 + (int)rank;            // this CTA's 128-row tile
    const int ucol = ct * BN + (int)rank * T::UH;    // first column of this CTA's half of U

    if (tid == 0) {
        for (int i = 0; i < T::NBAR; i++) mbar_init(&bars[i], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        *ok_sh = 1;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(2 * BN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    cluster_sync();   // barriers initialised and TMEM allocated in both CTAs
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (tid == 0) {
        bool ok = true;
        // this CTA's 128 rows of each component plane of L (columns of U)
        const __half *gl = Lpack + (size_t)(loff + rtile * TR) * KC;
        const __half *gu = Upack + (size_t)(uoff + ucol) * KC;
        constexpr uint32_t sbytes = sizeof(__half) * SUB, ubytes = sizeof(__half) * T::USUB;
        auto load = [&](int c) {
            __half *st = stage + (c % NSTAGE) * T::STAGE;
            mbar_expect_tx(&full[c % NSTAGE], 4 * (sbytes + ubytes));
            for (int comp = 0; comp < 4; comp++) {
                bulk_g2s(st + comp * SUB, gl + (size_t)(c * 4 + comp) * lpitch * KC, sbytes, &full[c % NSTAGE]);
                bulk_g2s(st + CHUNK_HALVES + comp * T::USUB, gu + (size_t)(c * 4 + comp) * upitch * KC, ubytes,
                         &full[c % NSTAGE]);
            }
        };
        for (int c = 0; c < NSTAGE && c < nchunk; c++) load(c);
        if (leader) {
            const uint32_t done_me = smem_u32(done), done_peer = peer_addr(done, 1);
            for (int c = 0; c < nchunk && ok; c++) {
                const int sidx = c % NSTAGE;
                const uint32_t par = (c / NSTAGE) & 1;
                if (!mbar_wait(&full[sidx], par, err) || !mbar_wait(&pfull[sidx], par, err)) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const __half *st = stage + sidx * T::STAGE;
                const uint64_t lrh = desc_sw64(st), lrl = desc_sw64(st + SUB), lih = desc_sw64(st + 2 * SUB),
                               lil = desc_sw64(st + 3 * SUB);
                const __half *su = st + CHUNK_HALVES;
                const uint64_t urh = desc_sw64(su), url = desc_sw64(su + T::USUB), uih = desc_sw64(su + 2 * T::USUB),
                               uil = desc_sw64(su + 3 * T::USUB);
                const uint32_t dre = tmem, dim = tmem + BN;
                constexpr uint32_t IDESC = Idesc<BN>::POS, IDESC_NEG_A = Idesc<BN>::NEG_A;
#pragma unroll
                for (int kk = 0; kk < KC / 16; kk++) {
                    const uint64_t a = (uint64_t)((kk * 32) >> 4);   // 16 fp16 = 32 bytes along K
                    const uint32_t acc0 = (c > 0 || kk > 0) ? 1u : 0u;
                    // Re += Lr Ur - Li Ui; small terms first, then the leading product
                    mma_pair(dre, lrl + a, urh + a, IDESC, acc0);
                    mma_pair(dre, lrh + a, url + a, IDESC, 1u);
                    mma_pair(dre, lil + a, uih + a, IDESC_NEG_A, 1u);
                    mma_pair(dre, lih + a, uil + a, IDESC_NEG_A, 1u);
                    mma_pair(dre, lih + a, uih + a, IDESC_NEG_A, 1u);
                    mma_pair(dre, lrh + a, urh + a, IDESC, 1u);
                    // Im += Lr Ui + Li Ur
                    mma_pair(dim, lrl + a, uih + a, IDESC, acc0);
                    mma_pair(dim, lrh + a, uil + a, IDESC, 1u);
                    mma_pair(dim, lil + a, urh + a, IDESC, 1u);
                    mma_pair(dim, lih + a, url + a, IDESC, 1u);
                    mma_pair(dim, lih + a, urh + a, IDESC, 1u);
                    mma_pair(dim, lrh + a, uih + a, IDESC, 1u);
                }
                // stage sidx is free in both CTAs once these MMAs have read it
                mma_commit(smem_u32(&empty[sidx]));
                mma_commit(peer_addr(&empty[sidx], 1));
                // refill the stage of chunk c - 1: its MMAs were queued ahead of chunk
                // c's, so waiting for them leaves chunk c's MMAs on the tensor pipe
                const int cp = c - 1;
                if (cp >= 0 && cp + NSTAGE < nchunk) {
                    if (!mbar_wait(&empty[cp % NSTAGE], (cp / NSTAGE) & 1, err)) { ok = false; break; }
                    load(cp + NSTAGE);
                }
            }
            // all MMAs of the pair done: both CTAs' accumulators are complete
            mma_commit(done_me);
            mma_commit(done_peer);
        } else {
            // the odd CTA: forward the arrival of each chunk to the even CTA's
            // barrier, refill a stage once the MMAs that read it are done
            const uint32_t pf0 = peer_addr(pfull, 0);
            for (int c = 0; c < nchunk && ok; c++) {
                const int sidx = c % NSTAGE;
                if (!mbar_wait(&full[sidx], (c / NSTAGE) & 1, err)) { ok = false; break; }
                mbar_arrive_remote(pf0 + 8u * (uint32_t)sidx);
                const int cp = c - 1;
                if (cp >= 0 && cp + NSTAGE < nchunk) {
                    if (!mbar_wait(&empty[cp % NSTAGE], (cp / NSTAGE) & 1, err)) { ok = false; break; }
                    load(cp + NSTAGE);
                }
            }
        }
        if (!ok) *ok_sh = 0;
    } else if (warp > 0) {
        // inverse column scales of the tile into shared memory
        for (int j = tid - 32; j < BN; j += 224) {
            const int col = c0 + ct * BN + j;
            col_is[j] = (col < c1) ? 1.f / pow2_scale(col_max(um, ld, col, krow / 64, (krow + K + 63) / 64)) : 0.f;
        }
        // C rows of this CTA into L2 while the MMAs run: (plane, row) segments
        const int ncol = min(BN, c1 - (c0 + ct * BN));
        const uint32_t bytes = (uint32_t)((ncol * 4 + 15) & ~15);
        for (int e = tid - 32; e < 2 * TR; e += 224) {
            const int pl = e / TR, rr = e % TR;
            const int row = r0 + rtile * TR + rr;
            if (row < r1 && ncol > 0) {
                const float *src = (pl ? Ai : Ar) + (size_t)row * ld + c0 + ct * BN;
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
        const int quarter = warp & 3;               // TMEM lanes 32 quarter ... (tcgen05.ld reach of this warp)
        const int pl = warp >> 2;                   // 0: real part, 1: imaginary part
        const int rowq = r0 + rtile * TR + quarter * 32;   // first row of this warp's 32
        const int ncol = c1 - (c0 + ct * BN);       // valid columns of this tile (may exceed BN)
        if (rowq < r1) {                            // warp-uniform
            const int row = rowq + lane;
            const float rs = row < r1 ? 1.f / pow2_scale(row_max(lm, row, nblk, kcol / 64, (kcol + K + 63) / 64)) : 0.f;
            const uint32_t tbase = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(pl * BN);
            // the stages are free once the MMAs are done: ER 4 KB tiles per warp
            constexpr int ER = T::ER;
            float *ring = reinterpret_cast<float *>(stage) + warp * ER * 1024;
            constexpr int NJ = BN / 32;
#pragma unroll 1
            for (int j = 0; j < NJ && j * 32 < ncol; j++) {
                uint32_t v[32];
                tmem_ld32(tbase + j * 32, v);
                float *tile = ring + (j % ER) * 1024;
                if (j >= ER) {   // the reduction that read this tile ER blocks ago is done with it
                    if (lane == 0) bulk_wait_read<ER - 1>();
                    __syncwarp();
                }
                // row `lane` of the tile; 16-byte chunk q sits at chunk q ^ (lane mod 8)
#pragma unroll
                for (int q = 0; q < 8; q++) {
                    const float4 cs = *reinterpret_cast<const float4 *>(col_is + j * 32 + 4 * q);
                    const float s0 = rs * cs.x, s1 = rs * cs.y, s2 = rs * cs.z, s3 = rs * cs.w;
                    float4 x;   // exact zeros outside the update (never 0 * inf)
                    x.x = s0 != 0.f ? -__uint_as_float(v[4 * q]) * s0 : 0.f;
                    x.y = s1 != 0.f ? -__uint_as_float(v[4 * q + 1]) * s1 : 0.f;
                    x.z = s2 != 0.f ? -__uint_as_float(v[4 * q + 2]) * s2 : 0.f;
                    x.w = s3 != 0.f ? -__uint_as_float(v[4 * q + 3]) * s3 : 0.f;
                    *reinterpret_cast<float4 *>(tile + lane * 32 + ((q ^ (lane & 7)) << 2)) = x;
                }
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // visible to the bulk copy
                __syncwarp();
                if (lane == 0) reduce_add_tile(&cmap, tile, c0 + ct * BN + j * 32, rowq, pl, f);
            }
            if (lane == 0) bulk_wait_read<0>();   // shared memory is read before the CTA exits
            __syncwarp();
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    // both CTAs are past every access to each other's shared memory and TMEM
    cluster_sync();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * BN));
    }
}

// ---------------------------------------------------------------------------
// Resident CTA pairs for the panel chain's K = 64 updates.  With K = 64 a
// tile's MMAs take a few microseconds while the fixed phases around them
// (cluster launch, TMEM allocation, first operand loads, the TMEM drain and
// the reductions) take longer.  Here each CTA pair stays resident and walks
// its tiles t = pair, pair + pairs, ... (256 x 128 tiles over every
// frequency of the update), with the phases of consecutive tiles overlapped:
//   * warp 0, lane 0 (both CTAs): producer -- the operand chunks of the next
//     tiles into a 3-stage ring as soon as the MMAs free a stage;
//   * warp 1, lane 0: the even CTA issues the MMAs of tile i into TMEM buffer
//     i mod 2 (two buffers of 256 columns: real and imaginary 128 x 128 per
//     CTA); the odd CTA forwards its chunk arrivals to the even CTA;
//   * warps 4-7 (both CTAs): epilogue -- drain buffer i mod 2 (lane quarter
//     warp - 4, real then imaginary part), scale, stage in shared memory and
//     reduce into C with bulk tensor reductions, then hand the buffer back to
//     the MMA thread (tempty, 4 arrivals from each CTA on the even CTA's
//     barrier), so the drain of tile i overlaps the MMAs of tile i + 1.
// The arithmetic per element is the kernel above's (same MMA order, same
// scaling), so the results are identical.  Every wait is bounded; a timeout
// marks every active frequency of the update failed and all roles stop.
// ---------------------------------------------------------------------------
constexpr int PBN = 128;
constexpr int PNST = 3;
using PT = Tile<PBN>;
constexpr int PNBAR = 3 * PNST + 4;                                  // full, empty, pfull, tfull[2], tempty[2]
constexpr int PEPI_FLOATS = 4 * 4 * 1024;                            // 4 warps x 4 staged 32 x 32 tiles
constexpr size_t PIPE_SMEM = sizeof(__half) * PNST * PT::STAGE + sizeof(float) * PEPI_FLOATS + 1024 +
                             8 * (PNBAR + 3) + sizeof(float) * 4 * 2 * PBN;

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(256, 1)
    k_update_tc_pipe(const __grid_constant__ CUtensorMap cmap, int N, int B, int r0, int r1, int c0, int c1,
                     int nchunk, const __half *__restrict__ Lpackb, size_t lstride, int lpitch, int loff,
                     const __half *__restrict__ Upackb, size_t ustride, int upitch, int uoff,
                     const float *__restrict__ lmaxb, const float *__restrict__ umaxb, size_t mstride, int nblk,
                     int kcol, int krow, int K, int ld, char *__restrict__ ctl, const int *__restrict__ active,
                     int tri_kb) {
    const int npr = (r1 - r0 + TM - 1) / TM, nct = (c1 - c0 + PBN - 1) / PBN;
    // tiles per frequency: the full npr x nct grid, or (lower-triangle mode,
    // tri_kb > 0) the tiles of row pair p with column tile < tri_cols(p)
    int per_f = npr * nct;
    if (tri_kb > 0) {
        per_f = 0;
        for (int p = 0; p < npr; p++) per_f += tri_cols(p, nct, tri_kb, PBN);
    }
    const int ntiles = per_f * B;
    auto tile_of = [&](int rr, int &rp, int &ct) {
        if (tri_kb <= 0) {
            rp = rr / nct;
            ct = rr - rp * nct;
            return;
        }
        rp = 0;
        while (rp < npr - 1) {
            const int nc = tri_cols(rp, nct, tri_kb, PBN);
            if (rr < nc) break;
            rr -= nc;
            rp++;
        }
        ct = rr;
    };
    const int pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;
    const uint32_t rank = cluster_rank();
    const bool leader = rank == 0;
    extern __shared__ uint8_t dyn_raw[];
    __half *stage = reinterpret_cast<__half *>((reinterpret_cast<uintptr_t>(dyn_raw) + 1023) & ~(uintptr_t)1023);
    float *epi = reinterpret_cast<float *>(stage + PNST * PT::STAGE);
    uint64_t *bars = reinterpret_cast<uint64_t *>(epi + PEPI_FLOATS);
    uint64_t *full = bars, *empty = bars + PNST, *pfull = bars + 2 * PNST, *tfull = bars + 3 * PNST,
             *tempty = tfull + 2;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + PNBAR);
    volatile int *abort_sh = reinterpret_cast<volatile int *>(tmem_slot + 1);
    // [epilogue warp][2][PBN] inverse column scales (16-byte aligned)
    float *colsc = reinterpret_cast<float *>(bars + PNBAR + 3);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    auto errp = [&](int f) { return reinterpret_cast<int *>(ctl + 64 * f + 36); };
    auto fail_all = [&]() {
        *abort_sh = 1;
        for (int f = 0; f < B; f++)
            if (active[f]) atomicExch(errp(f), 3);
    };

    if (tid == 0) {
        for (int i = 0; i < PNBAR; i++) mbar_init(&bars[i], i >= 3 * PNST + 2 ? 8 : 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        *abort_sh = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(4 * PBN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    cluster_sync();   // barriers initialised and TMEM allocated in both CTAs
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        // producer
        constexpr uint32_t sbytes = sizeof(__half) * SUB, ubytes = sizeof(__half) * PT::USUB;
        long long g = 0;
        for (int t = pair; t < ntiles && !*abort_sh; t += npairs) {
            const int f = t / per_f;
            int rp, ct;
            tile_of(t - f * per_f, rp, ct);
            if (!active[f]) continue;
            const __half *gl = Lpackb + lstride * f + (size_t)(loff + (rp * 2 + (int)rank) * TR) * KC;
            const __half *gu = Upackb + ustride * f + (size_t)(uoff + ct * PBN + (int)rank * PT::UH) * KC;
            for (int c = 0; c < nchunk; c++, g++) {
                const int sidx = (int)(g % PNST);
                if (g >= PNST && !mbar_wait(&empty[sidx], (uint32_t)((g / PNST - 1) & 1), errp(f))) {
                    fail_all();
                    break;
                }
                __half *st = stage + sidx * PT::STAGE;
                mbar_expect_tx(&full[sidx], 4 * (sbytes + ubytes));
                for (int comp = 0; comp < 4; comp++) {
                    bulk_g2s(st + comp * SUB, gl + (size_t)(c * 4 + comp) * lpitch * KC, sbytes, &full[sidx]);
                    bulk_g2s(st + CHUNK_HALVES + comp * PT::USUB, gu + (size_t)(c * 4 + comp) * upitch * KC, ubytes,
                             &full[sidx]);
                }
            }
        }
    } else if (warp == 1 && lane == 0 && leader) {
        // MMA issuer
        const uint32_t tf_peer = peer_addr(tfull, 1);
        long long g = 0;
        int i = 0;
        for (int t = pair; t < ntiles && !*abort_sh; t += npairs) {
            const int f = t / per_f;
            if (!active[f]) continue;
            const int b = i & 1;
            if (!mbar_wait(&tempty[b], (uint32_t)(((i >> 1) & 1) ^ 1), errp(f))) {
                fail_all();
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t dre = tmem + (uint32_t)(b * 2 * PBN), dim = dre + PBN;
            bool ok = true;
            for (int c = 0; c < nchunk; c++, g++) {
                const int sidx = (int)(g % PNST);
                const uint32_t par = (uint32_t)((g / PNST) & 1);
                if (!mbar_wait(&full[sidx], par, errp(f)) || !mbar_wait(&pfull[sidx], par, errp(f))) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const __half *st = stage + sidx * PT::STAGE;
                const uint64_t lrh = desc_sw64(st), lrl = desc_sw64(st + SUB), lih = desc_sw64(st + 2 * SUB),
                               lil = desc_sw64(st + 3 * SUB);
                const __half *su = st + CHUNK_HALVES;
                const uint64_t urh = desc_sw64(su), url = desc_sw64(su + PT::USUB),
                               uih = desc_sw64(su + 2 * PT::USUB), uil = desc_sw64(su + 3 * PT::USUB);
                constexpr uint32_t IDESC = Idesc<PBN>::POS, IDESC_NEG_A = Idesc<PBN>::NEG_A;
#pragma unroll
                for (int kk = 0; kk < KC / 16; kk++) {
                    const uint64_t a = (uint64_t)((kk * 32) >> 4);
                    const uint32_t acc0 = (c > 0 || kk > 0) ? 1u : 0u;
                    mma_pair(dre, lrl + a, urh + a, IDESC, acc0);
                    mma_pair(dre, lrh + a, url + a, IDESC, 1u);
                    mma_pair(dre, lil + a, uih + a, IDESC_NEG_A, 1u);
                    mma_pair(dre, lih + a, uil + a, IDESC_NEG_A, 1u);
                    mma_pair(dre, lih + a, uih + a, IDESC_NEG_A, 1u);
                    mma_pair(dre, lrh + a, urh + a, IDESC, 1u);
                    mma_pair(dim, lrl + a, uih + a, IDESC, acc0);
                    mma_pair(dim, lrh + a, uil + a, IDESC, 1u);
                    mma_pair(dim, lil + a, urh + a, IDESC, 1u);
                    mma_pair(dim, lih + a, url + a, IDESC, 1u);
                    mma_pair(dim, lih + a, urh + a, IDESC, 1u);
                    mma_pair(dim, lrh + a, uih + a, IDESC, 1u);
                }
                mma_commit(smem_u32(&empty[sidx]));
                mma_commit(peer_addr(&empty[sidx], 1));
            }
            if (!ok) {
                fail_all();
                break;
            }
            // buffer b complete in both CTAs
            mma_commit(smem_u32(&tfull[b]));
            mma_commit(tf_peer + 8u * (uint32_t)b);
            i++;
        }
    } else if (warp == 1 && lane == 0) {
        // the odd CTA: forward the arrival of each chunk to the even CTA
        const uint32_t pf0 = peer_addr(pfull, 0);
        long long g = 0;
        for (int t = pair; t < ntiles && !*abort_sh; t += npairs) {
            const int f = t / per_f;
            if (!active[f]) continue;
            bool ok = true;
            for (int c = 0; c < nchunk; c++, g++) {
                const int sidx = (int)(g % PNST);
                if (!mbar_wait(&full[sidx], (uint32_t)((g / PNST) & 1), errp(f))) {
                    ok = false;
                    break;
                }
                mbar_arrive_remote(pf0 + 8u * (uint32_t)sidx);
            }
            if (!ok) {
                fail_all();
                break;
            }
        }
    } else if (warp >= 4) {
        // epilogue: lane quarter q of the TMEM accumulators
        const int q = warp - 4;
        const uint32_t te0 = peer_addr(tempty, 0);
        float *ring = epi + q * 4 * 1024;
        float *wcs = colsc + q * 2 * PBN;   // this warp's copy: no barrier across the epilogue warps
        int staged = 0, i = 0;
        for (int t = pair; t < ntiles && !*abort_sh; t += npairs) {
            const int f = t / per_f;
            int rp, ct;
            tile_of(t - f * per_f, rp, ct);
            if (!active[f]) continue;
            const int b = i & 1;
            const float *lm = lmaxb + mstride * f, *um = umaxb + mstride * f;
            // inverse column scales of this tile (the warp's slot b, read last by tile i - 2)
            for (int e = lane; e < PBN; e += 32) {
                const int col = c0 + ct * PBN + e;
                wcs[b * PBN + e] =
                    col < c1 ? 1.f / pow2_scale(col_max(um, ld, col, krow / 64, (krow + K + 63) / 64)) : 0.f;
            }
            __syncwarp();
            bool have = mbar_wait(&tfull[b], (uint32_t)((i >> 1) & 1), errp(f));
            have = __all_sync(0xffffffffu, have);
            if (!have) {
                if (lane == 0) fail_all();
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int rowq = r0 + (rp * 2 + (int)rank) * TR + q * 32;
            const int ncol = c1 - (c0 + ct * PBN);
            if (rowq < r1) {   // warp-uniform
                const int row = rowq + lane;
                const float rs =
                    row < r1 ? 1.f / pow2_scale(row_max(lm, row, nblk, kcol / 64, (kcol + K + 63) / 64)) : 0.f;
#pragma unroll 1
                for (int pl = 0; pl < 2; pl++) {
                    const uint32_t tbase = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * 2 * PBN + pl * PBN);
#pragma unroll 1
                    for (int j = 0; j < PBN / 32 && j * 32 < ncol; j++) {
                        uint32_t v[32];
                        tmem_ld32(tbase + j * 32, v);
                        float *tile = ring + (staged & 3) * 1024;
                        if (staged >= 4) {   // the reduction that read this tile four tiles ago is done with it
                            if (lane == 0) bulk_wait_read<3>();
                            __syncwarp();
                        }
#pragma unroll
                        for (int qq = 0; qq < 8; qq++) {
                            const float4 cs = *reinterpret_cast<const float4 *>(wcs + b * PBN + j * 32 + 4 * qq);
                            const float s0 = rs * cs.x, s1 = rs * cs.y, s2 = rs * cs.z, s3 = rs * cs.w;
                            float4 x;
                            x.x = s0 != 0.f ? -__uint_as_float(v[4 * qq]) * s0 : 0.f;
                            x.y = s1 != 0.f ? -__uint_as_float(v[4 * qq + 1]) * s1 : 0.f;
                            x.z = s2 != 0.f ? -__uint_as_float(v[4 * qq + 2]) * s2 : 0.f;
                            x.w = s3 != 0.f ? -__uint_as_float(v[4 * qq + 3]) * s3 : 0.f;
                            *reinterpret_cast<float4 *>(tile + lane * 32 + ((qq ^ (lane & 7)) << 2)) = x;
                        }
                        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                        __syncwarp();
                        if (lane == 0) reduce_add_tile(&cmap, tile, c0 + ct * PBN + j * 32, rowq, pl, f);
                        staged++;
                    }
                }
            }
            // buffer b drained in this CTA: hand it back to the MMA thread
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive_remote(te0 + 8u * (uint32_t)b);
            i++;
        }
        if (lane == 0) bulk_wait_read<0>();   // shared memory is read before the CTA exits
        __syncwarp();
    }
    __syncthreads();
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    cluster_sync();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(4 * PBN));
    }
}

}  // namespace

static bool g_tc_disabled = false;

efie_status efie_tc_attrs() {
    static bool done = false;
    if (done) return EFIE_OK;
    EFIE_CUDA(cudaFuncSetAttribute(k_update_tc<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)Tile<256>::SMEM));
    EFIE_CUDA(cudaFuncSetAttribute(k_update_tc<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)Tile<128>::SMEM));
    EFIE_CUDA(cudaFuncSetAttribute(k_update_tc<128>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    EFIE_CUDA(cudaFuncSetAttribute(k_update_tc_pipe, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PIPE_SMEM));
    done = true;
    return EFIE_OK;
}

extern "C" void efie_debug_disable_tensor_cores(int disable) { g_tc_disabled = disable != 0; }

efie_status efie_encode_tiled(void *map, CUtensorMapDataType type, int rank, void *base, const cuuint64_t *dims,
                              const cuuint64_t *strides, const cuuint32_t *box, CUtensorMapSwizzle swizzle) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        EFIE_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !fn)
            return efie_fail(EFIE_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    const CUresult r = encode(reinterpret_cast<CUtensorMap *>(map), type, (cuuint32_t)rank, base, dims, strides, box,
                              estr, CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return efie_fail(EFIE_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    return EFIE_OK;
}

namespace {
// the planes of every frequency slot as one float tensor [B][2][N][ld]
// (innermost first: column, row, plane, slot), 32 x 32 boxes, 128B swizzle
efie_status encode_planes_map(SolveWork &w) {
    const cuuint64_t dims[4] = {(cuuint64_t)w.N, (cuuint64_t)w.N, 2, (cuuint64_t)w.B};
    const cuuint64_t strides[3] = {sizeof(float) * (cuuint64_t)w.ld, sizeof(float) * (cuuint64_t)w.ld * w.N,
                                   sizeof(float) * (cuuint64_t)w.pstride};
    const cuuint32_t box[4] = {32, 32, 1, 1};
    return efie_encode_tiled(w.planes_map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, w.planes.p, dims, strides, box,
                             CU_TENSOR_MAP_SWIZZLE_128B);
}

// halves per frequency slot of a packed panel with `nchunk` K chunks
size_t pack_stride(const SolveWork &w, int nchunk) { return (size_t)nchunk * 4 * w.ppitch * KC; }
}  // namespace

// Staging for the packed panels of an N x N LU (per frequency slot), the
// planes' tensor map and the kernel attributes: done when the workspace is
// created (after the planes), so that the factor sequence allocates nothing
// and can be captured into a CUDA graph.  A panel's pitch leaves room for the
// 256 rows a CTA pair may read past the last row of a view.
efie_status efie_gemm_workspace(SolveWork &w) {
    EFIE_TRY(efie_tc_attrs());
    EFIE_TRY(encode_planes_map(w));
    w.ppitch = (w.N + 256 + TR - 1) / TR * TR;
    const size_t outer = sizeof(__half) * pack_stride(w, NCHUNK_MAX) * w.B;
    const size_t inpanel = sizeof(__half) * pack_stride(w, 64 / KC) * w.B;
    for (int i = 0; i < 2; i++) {
        EFIE_TRY(w.packL[i].reserve(outer));
        EFIE_TRY(w.packU[i].reserve(outer));
    }
    EFIE_TRY(w.ipL.reserve(inpanel));
    EFIE_TRY(w.ipU.reserve(inpanel));
    return EFIE_OK;
}

PackView efie_inpanel_view(const SolveWork &w, bool lower) {
    PackView v;
    v.base = (lower ? w.ipL : w.ipU).p;
    v.stride = pack_stride(w, 64 / KC);
    v.pitch = w.ppitch;
    return v;
}

efie_status efie_pack_l(efie_ctx *ctx, SolveWork &w, DevBuf &buf, int r0, int r1, int kcol, int K, PackView *out) {
    if (K <= 0 || K > KMAX || r1 <= r0) return efie_fail(EFIE_ERR_ARGS, "efie_pack_l: bad block");
    const int nchunk = (K + KC - 1) / KC;
    const size_t stride = pack_stride(w, nchunk);
    if (buf.bytes < sizeof(__half) * stride * w.B) return efie_fail(EFIE_ERR_ARGS, "efie_pack_l: staging too small");
    cudaStream_t st = ctx->stream;
    size_t tok = ctx->log.begin(st);
    k_pack_l<<<dim3((r1 - r0 + TR - 1) / TR, nchunk, w.B), 256, 0, st>>>(
        w.N, r0, r1, kcol, K, w.ppitch, w.planes.as<float>(), w.pstride, w.ld, w.lmax.as<float>(), w.mstride, w.nblk,
        buf.as<__half>(), stride, w.active.as<int>());
    EFIE_CUDA(cudaGetLastError());
    ctx->log.end(EFIE_K_PANEL, st, tok, 0.0, 1);
    *out = PackView{buf.p, stride, w.ppitch, 0};
    return EFIE_OK;
}

efie_status efie_pack_u(efie_ctx *ctx, SolveWork &w, DevBuf &buf, int c0, int c1, int krow, int K, PackView *out) {
    if (K <= 0 || K > KMAX || c1 <= c0) return efie_fail(EFIE_ERR_ARGS, "efie_pack_u: bad block");
    const int nchunk = (K + KC - 1) / KC;
    const size_t stride = pack_stride(w, nchunk);
    if (buf.bytes < sizeof(__half) * stride * w.B) return efie_fail(EFIE_ERR_ARGS, "efie_pack_u: staging too small");
    cudaStream_t st = ctx->stream;
    size_t tok = ctx->log.begin(st);
    k_pack_u<<<dim3((c1 - c0 + TR - 1) / TR, nchunk, w.B), 256, 0, st>>>(
        w.N, c0, c1, krow, K, w.ppitch, w.planes.as<float>(), w.pstride, w.ld, w.umax.as<float>(), w.mstride,
        buf.as<__half>(), stride, w.active.as<int>());
    EFIE_CUDA(cudaGetLastError());
    ctx->log.end(EFIE_K_PANEL, st, tok, 0.0, 1);
    *out = PackView{buf.p, stride, w.ppitch, 0};
    return EFIE_OK;
}

bool efie_gemm_uses_tc(int rows, int cols, int K) {
    return !g_tc_disabled && K > 0 && K <= KMAX && rows >= 64 && cols >= 64;
}

// C[r0:r1, c0:c1] -= L[r0:r1, kcol:kcol+K] * U[krow:krow+K, c0:c1] for every
// active frequency: tensor cores from the packed views when the block spans
// enough work, CUDA cores from the factors otherwise.
efie_status efie_gemm_update(efie_ctx *ctx, SolveWork &w, int r0, int r1, int c0, int c1, int kcol, int krow, int K,
                             int nact, const PackView &Lv, const PackView &Uv, int tri_kb) {
    const int rows = r1 - r0, cols = c1 - c0;
    if (rows <= 0 || cols <= 0 || K <= 0) return EFIE_OK;
    if (tri_kb > 0 && (r0 != c0 || r1 != c1 || tri_kb % 64))
        return efie_fail(EFIE_ERR_ARGS, "efie_gemm_update: the lower-triangle mode takes a square block");
    if (!efie_gemm_uses_tc(rows, cols, K)) {
        for (int k0 = 0; k0 < K; k0 += 64)
            EFIE_TRY(efie_update_simt(ctx, w, r0, r1, c0, c1, kcol + k0, krow + k0, std::min(64, K - k0), nact));
        return EFIE_OK;
    }
    // resident pairs: the chain's K = 64 updates, and of the outer panels'
    // updates the rectangular ones (the strip of the next panel on the
    // critical path; the lower-triangle bulk runs beside the chain on the
    // one-tile kernel, whose short-lived pairs leave the chain its SMs)
    if (K <= 64 ? w.resident_chain : (w.resident_bulk && tri_kb == 0)) {
        // resident, pipelined CTA pairs over 256 x 128 tiles
        if (!Lv.base || !Uv.base || (Lv.off & 7) || (Uv.off & 7) ||
            Lv.off + (rows + TM - 1) / TM * TM > Lv.pitch || Uv.off + (cols + PBN - 1) / PBN * PBN > Uv.pitch)
            return efie_fail(EFIE_ERR_ARGS, "efie_gemm_update: packed operands do not cover the block");
        EFIE_TRY(efie_tc_attrs());
        cudaStream_t st = ctx->stream;
        const int npr = (rows + TM - 1) / TM, nct = (cols + PBN - 1) / PBN;
        long long per_f = (long long)npr * nct;
        double entries = (double)rows * cols;
        if (tri_kb > 0) {
            per_f = 0;
            for (int p = 0; p < npr; p++) per_f += tri_cols(p, nct, tri_kb, PBN);
            entries = 0;
            for (int q0 = 0; q0 < rows; q0 += tri_kb)
                entries += (double)std::min(tri_kb, rows - q0) * std::min(cols, q0 + tri_kb);
        }
        // the outer panels' updates run beside the panel chain (look-ahead
        // streams): resident pairs would hold every SM for the whole update, so
        // they leave 16 SMs to the chain's kernels
        const int avail = K <= 64 ? ctx->num_sms / 2 : ctx->num_sms / 2 - 8;
        const int pairs = (int)std::min<long long>(std::max(1, avail), per_f * w.B);
        size_t tok = ctx->log.begin(st);
        k_update_tc_pipe<<<2 * pairs, 256, PIPE_SMEM, st>>>(
            *reinterpret_cast<const CUtensorMap *>(w.planes_map), w.N, w.B, r0, r1, c0, c1, (K + KC - 1) / KC,
            static_cast<const __half *>(Lv.base), Lv.stride, Lv.pitch, Lv.off, static_cast<const __half *>(Uv.base),
            Uv.stride, Uv.pitch, Uv.off, w.lmax.as<float>(), w.umax.as<float>(), w.mstride, w.nblk, kcol, krow, K,
            w.ld, w.ctl.as<char>(), w.active.as<int>(), tri_kb);
        EFIE_CUDA(cudaGetLastError());
        ctx->log.end(EFIE_K_GEMM, st, tok, 8.0 * entries * K * nact);
        return EFIE_OK;
    }
    // tile width of the pair: the panel chain's K = 64 updates and the outer
    // panels' updates each have their own (tuned) choice
    const int BN = K <= 64 ? w.tn_chain : w.tn_bulk;
    if (BN != 256 && BN != 128) return efie_fail(EFIE_ERR_ARGS, "efie_gemm_update: tile width must be 128 or 256");
    if (!Lv.base || !Uv.base || (Lv.off & 7) || (Uv.off & 7) ||
        Lv.off + (rows + TM - 1) / TM * TM > Lv.pitch || Uv.off + (cols + BN - 1) / BN * BN > Uv.pitch)
        return efie_fail(EFIE_ERR_ARGS, "efie_gemm_update: packed operands do not cover the block");
    EFIE_TRY(efie_tc_attrs());
    const int N = w.N, B = w.B;
    cudaStream_t st = ctx->stream;
    const int npr = (rows + TM - 1) / TM, nct = (cols + BN - 1) / BN;   // 256-row pairs, BN-column tiles
    const int nchunk = (K + KC - 1) / KC;
    // work: the entries the update must produce (in the lower-triangle mode
    // those of column blocks <= row block, not the tiles' overhang)
    dim3 grid(2 * nct, npr, B);
    double entries = (double)rows * cols;
    if (tri_kb > 0) {
        int ntiles = 0;
        for (int p = 0; p < npr; p++) ntiles += tri_cols(p, nct, tri_kb, BN);
        grid = dim3(2 * ntiles, 1, B);
        entries = 0;
        for (int q0 = 0; q0 < rows; q0 += tri_kb)
            entries += (double)std::min(tri_kb, rows - q0) * std::min(cols, q0 + tri_kb);
    }
    size_t tok = ctx->log.begin(st);
    const CUtensorMap &cm = *reinterpret_cast<const CUtensorMap *>(w.planes_map);
    const __half *lb = static_cast<const __half *>(Lv.base), *ub = static_cast<const __half *>(Uv.base);
    if (BN == 256)
        k_update_tc<256><<<grid, 256, Tile<256>::SMEM, st>>>(
            cm, N, r0, r1, c0, c1, nchunk, lb, Lv.stride, Lv.pitch, Lv.off, ub, Uv.stride, Uv.pitch, Uv.off,
            w.lmax.as<float>(), w.umax.as<float>(), w.mstride, w.nblk, kcol, krow, K, w.planes.as<float>(),
            w.pstride, w.ld, w.ctl.as<char>(), w.active.as<int>(), tri_kb);
    else
        k_update_tc<128><<<grid, 256, Tile<128>::SMEM, st>>>(
            cm, N, r0, r1, c0, c1, nchunk, lb, Lv.stride, Lv.pitch, Lv.off, ub, Uv.stride, Uv.pitch, Uv.off,
            w.lmax.as<float>(), w.umax.as<float>(), w.mstride, w.nblk, kcol, krow, K, w.planes.as<float>(),
            w.pstride, w.ld, w.ctl.as<char>(), w.active.as<int>(), tri_kb);
    EFIE_CUDA(cudaGetLastError());
    ctx->log.end(EFIE_K_GEMM, st, tok, 8.0 * entries * K * nact);
    return EFIE_OK;
}
