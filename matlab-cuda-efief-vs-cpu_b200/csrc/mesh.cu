// The two-plate mesh and its RWG topology built on the GPU
// (make_patch_with_ground_mesh.m:1-46, build_rwg_interior.m:1-113,
// pick_port_edge_by_point_and_layer.m:1-11), so that a design family can be
// meshed without MATLAB or a host pass over the faces.
//
// RWG numbering must stay bit-exact: the reference numbers the interior edges
// in the lexicographic order of unique(sort(edge),'rows') (:25) and takes the
// first incidence in (triangle, local edge) order as the plus side (:47-63).
// Here the 3 Nt directed edges are bucketed by their lower vertex (counting
// sort), each bucket is sorted by (higher vertex, raw row) -- a handful of
// entries per vertex -- and the buckets are walked in vertex order: that is
// the lexicographic order of (lo, hi) with the raw order inside a group, as a
// stable sort would give, without a global sort.  Floating-point outputs use
// explicitly rounded operations in the reference's order (no FMA
// contraction), so they are bit-identical to the host producers.
#include <algorithm>
#include <cmath>
#include <vector>

#include "efie_internal.h"

namespace {

__device__ __forceinline__ double ad(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sb(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ml(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double norm3(double x, double y, double z) {
    return __dsqrt_rn(ad(ad(ml(x, x), ml(y, y)), ml(z, z)));
}

// MATLAB linspace(d1, d2, n): d1 + (i (d2 - d1)) / (n - 1), both ends pinned
__device__ __forceinline__ double linspace_at(double d1, double d2, int n, int i) {
    if (i == 0) return d1;
    if (i == n - 1) return d2;
    return ad(d1, __ddiv_rn(ml((double)i, sb(d2, d1)), (double)(n - 1)));
}

struct Plate {
    double W, L, z;
    int nx, ny;
    int voff, toff;
};

// make_patch_with_ground_mesh.m:5-7 / :23-25 (vertices) and :9-20 / :27-39
// (faces, two per rectangle split along (v1, v4)); vertex_order 0 numbers the
// vertices y-fastest as meshgrid(:) does, 1 x-fastest like the faces.
__global__ void k_mesh(Plate P0, Plate P1, int Nv, int Nt, int vertex_order, double *__restrict__ V,
                       int *__restrict__ F) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    const int plate = blockIdx.y;
    const Plate P = plate == 0 ? P0 : P1;
    const int nvp = (P.nx + 1) * (P.ny + 1);
    if (idx < nvp) {
        int i, j;   // x and y grid indices of this vertex
        if (vertex_order == 0) j = idx % (P.ny + 1), i = idx / (P.ny + 1);
        else i = idx % (P.nx + 1), j = idx / (P.nx + 1);
        const int vi = P.voff + idx;
        V[vi] = linspace_at(-P.W / 2, P.W / 2, P.nx + 1, i);
        V[vi + Nv] = linspace_at(-P.L / 2, P.L / 2, P.ny + 1, j);
        V[vi + 2 * (size_t)Nv] = P.z;
    }
    if (idx < P.nx * P.ny) {
        const int i = idx % P.nx + 1, j = idx / P.nx + 1;
        const int v1 = P.voff + (j - 1) * (P.nx + 1) + i, v2 = v1 + 1, v3 = v1 + (P.nx + 1), v4 = v3 + 1;
        const int t = P.toff + 2 * idx;
        F[t] = v1; F[t + Nt] = v2; F[t + 2 * (size_t)Nt] = v4;
        F[t + 1] = v1; F[t + 1 + Nt] = v4; F[t + 1 + 2 * (size_t)Nt] = v3;
    }
}

// raw directed edge r = 3 t + le: (F(t, le), F(t, le + 1)) (build_rwg_interior.m:10-23)
__device__ __forceinline__ void raw_edge(const int *F, int Nt, int r, int &a, int &b) {
    const int t = r / 3, le = r - 3 * t;
    a = F[t + (size_t)le * Nt];
    b = F[t + (size_t)((le + 1) % 3) * Nt];
}

__global__ void k_raw_count(int Nv, int Nt, const int *__restrict__ F, int *__restrict__ cnt, int *__restrict__ bad) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= 3 * Nt) return;
    int a, b;
    raw_edge(F, Nt, r, a, b);
    if (a < 1 || a > Nv || b < 1 || b > Nv) {
        atomicExch(bad, 1);
        return;
    }
    atomicAdd(&cnt[min(a, b) - 1], 1);
}

__global__ void k_raw_scatter(int Nv, int Nt, const int *__restrict__ F, const int *__restrict__ off,
                              int *__restrict__ fill, int *__restrict__ bucket) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= 3 * Nt) return;
    int a, b;
    raw_edge(F, Nt, r, a, b);
    if (a < 1 || a > Nv || b < 1 || b > Nv) return;
    const int lo = min(a, b) - 1;
    bucket[off[lo] + atomicAdd(&fill[lo], 1)] = r;
}

// Sort the bucket of vertex v by (higher vertex, raw row) and count its
// interior edges (groups of exactly two incidences, build_rwg_interior.m:29-30).
__global__ void k_bucket_sort(int Nv, int Nt, const int *__restrict__ F, const int *__restrict__ off,
                              int *__restrict__ bucket, int *__restrict__ icnt) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= Nv) return;
    const int s0 = off[v], s1 = off[v + 1];
    auto key = [&](int r) -> long long {
        int a, b;
        raw_edge(F, Nt, r, a, b);
        return ((long long)max(a, b) << 32) | (long long)r;
    };
    for (int i = s0 + 1; i < s1; i++) {
        const int r = bucket[i];
        const long long k = key(r);
        int j = i - 1;
        while (j >= s0 && key(bucket[j]) > k) {
            bucket[j + 1] = bucket[j];
            j--;
        }
        bucket[j + 1] = r;
    }
    int n = 0;
    for (int s = s0; s < s1;) {
        const long long hs = key(bucket[s]) >> 32;
        int e = s + 1;
        while (e < s1 && (key(bucket[e]) >> 32) == hs) e++;
        if (e - s == 2) n++;
        s = e;
    }
    icnt[v] = n;
}

// Exclusive prefix sum over n counts (one CTA); out[n] = total.
__global__ void __launch_bounds__(1024) k_scan(int n, const int *__restrict__ cnt, int *__restrict__ out) {
    __shared__ int part[1024];
    const int tid = threadIdx.x;
    const int per = (n + 1023) / 1024;
    const int b0 = min(n, tid * per), b1 = min(n, b0 + per);
    int s = 0;
    for (int i = b0; i < b1; i++) s += cnt[i];
    part[tid] = s;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const int v = tid >= o ? part[tid - o] : 0;
        __syncthreads();
        part[tid] += v;
        __syncthreads();
    }
    int run = tid ? part[tid - 1] : 0;
    for (int i = b0; i < b1; i++) {
        out[i] = run;
        run += cnt[i];
    }
    if (tid == 1023) out[n] = part[1023];
}

// zmid = (max z + min z) / 2 over the vertices (build_rwg_interior.m:88), one CTA
__global__ void __launch_bounds__(1024) k_zmid(int Nv, const double *__restrict__ V, double *__restrict__ zmid) {
    __shared__ double lo[1024], hi[1024];
    const int tid = threadIdx.x;
    double a = V[2 * (size_t)Nv], b = a;
    for (int i = tid; i < Nv; i += 1024) {
        const double z = V[i + 2 * (size_t)Nv];
        a = fmin(a, z);
        b = fmax(b, z);
    }
    lo[tid] = a;
    hi[tid] = b;
    __syncthreads();
    for (int o = 512; o > 0; o >>= 1) {
        if (tid < o) {
            lo[tid] = fmin(lo[tid], lo[tid + o]);
            hi[tid] = fmax(hi[tid], hi[tid + o]);
        }
        __syncthreads();
    }
    if (tid == 0) *zmid = ml(0.5, ad(hi[0], lo[0]));
}

struct RwgOut {
    int *edge, *plusTri, *minusTri, *plusSign, *minusSign, *zSign;
    double *rp, *rm, *Ap, *Am, *len, *center;
};

// RWG arrays of the interior edges of vertex v's bucket (build_rwg_interior.m:47-113)
__global__ void k_rwg_fill(int Nv, int Nt, int Ne, const double *__restrict__ V, const int *__restrict__ F,
                           const int *__restrict__ off, const int *__restrict__ bucket, const int *__restrict__ eoff,
                           const double *__restrict__ zmid_p, RwgOut o, int *__restrict__ bad) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= Nv) return;
    const double zmid = *zmid_p;
    const int s0 = off[v], s1 = off[v + 1];
    int e = eoff[v];
    auto hi_of = [&](int r) {
        int a, b;
        raw_edge(F, Nt, r, a, b);
        return max(a, b);
    };
    auto vtx = [&](int id, double *r) {
        r[0] = V[id - 1];
        r[1] = V[id - 1 + Nv];
        r[2] = V[id - 1 + 2 * (size_t)Nv];
    };
    for (int s = s0; s < s1;) {
        const int hs = hi_of(bucket[s]);
        int t = s + 1;
        while (t < s1 && hi_of(bucket[t]) == hs) t++;
        if (t - s == 2) {
            const int r1 = bucket[s], r2 = bucket[s + 1];   // first and second incidence (raw order)
            int a1, b1, a2, b2;
            raw_edge(F, Nt, r1, a1, b1);
            raw_edge(F, Nt, r2, a2, b2);
            const int a = v + 1, b = hs;
            o.edge[e] = a;
            o.edge[e + Ne] = b;
            o.plusTri[e] = r1 / 3 + 1;
            o.minusTri[e] = r2 / 3 + 1;
            o.plusSign[e] = (a1 == a && b1 == b) ? 1 : -1;    // :50-63
            o.minusSign[e] = (a2 == a && b2 == b) ? 1 : -1;
            double ra[3], rb[3];
            vtx(a, ra);
            vtx(b, rb);
            o.len[e] = norm3(sb(rb[0], ra[0]), sb(rb[1], ra[1]), sb(rb[2], ra[2]));   // :75
            double c[3];
            for (int k = 0; k < 3; k++) {
                c[k] = ml(0.5, ad(ra[k], rb[k]));
                o.center[e + (size_t)k * Ne] = c[k];
            }
            o.zSign[e] = c[2] > zmid ? 1 : -1;                // :89-90
            for (int side = 0; side < 2; side++) {            // :80-84, :108-112
                const int tri = (side == 0 ? r1 : r2) / 3;
                const int tv[3] = {F[tri], F[tri + Nt], F[tri + 2 * (size_t)Nt]};
                int opp = 0, nopp = 0;
                for (int k = 0; k < 3; k++)
                    if (tv[k] != a && tv[k] != b) opp = tv[k], nopp++;
                if (nopp != 1) {
                    atomicExch(bad, 2);
                    continue;
                }
                double p1[3], p2[3], p3[3], ro[3];
                vtx(tv[0], p1);
                vtx(tv[1], p2);
                vtx(tv[2], p3);
                vtx(opp, ro);
                const double e1x = sb(p2[0], p1[0]), e1y = sb(p2[1], p1[1]), e1z = sb(p2[2], p1[2]);
                const double e2x = sb(p3[0], p1[0]), e2y = sb(p3[1], p1[1]), e2z = sb(p3[2], p1[2]);
                const double cx = sb(ml(e1y, e2z), ml(e1z, e2y)), cy = sb(ml(e1z, e2x), ml(e1x, e2z)),
                             cz = sb(ml(e1x, e2y), ml(e1y, e2x));
                const double A = ml(0.5, norm3(cx, cy, cz));
                double *dst = side == 0 ? o.rp : o.rm;
                for (int k = 0; k < 3; k++) dst[e + (size_t)k * Ne] = ro[k];
                (side == 0 ? o.Ap : o.Am)[e] = A;
            }
            e++;
        }
        s = t;
    }
}

// pick_port_edge_by_point_and_layer.m:2-10: the first edge of the layer at
// the smallest centre distance (min keeps the first minimum), one CTA.
__global__ void __launch_bounds__(1024) k_pick_port(int Ne, const double *__restrict__ center,
                                                    const int *__restrict__ zSign, double px, double py, double pz,
                                                    int layer, int *__restrict__ eidx) {
    __shared__ double bd[1024];
    __shared__ int be[1024];
    const int tid = threadIdx.x;
    double best = 0.0;
    int arg = -1;
    for (int e = tid; e < Ne; e += 1024) {
        if (zSign[e] != layer) continue;
        const double d = norm3(sb(center[e], px), sb(center[e + Ne], py), sb(center[e + 2 * (size_t)Ne], pz));
        if (arg < 0 || d < best) best = d, arg = e;
    }
    bd[tid] = best;
    be[tid] = arg;
    __syncthreads();
    for (int o = 512; o > 0; o >>= 1) {
        if (tid < o) {
            const int e2 = be[tid + o];
            if (e2 >= 0 && (be[tid] < 0 || bd[tid + o] < bd[tid] || (bd[tid + o] == bd[tid] && e2 < be[tid])))
                bd[tid] = bd[tid + o], be[tid] = e2;
        }
        __syncthreads();
    }
    if (tid == 0) *eidx = be[0] + 1;   // 0: no edge on the layer
}

}  // namespace

struct efie_design {
    efie_ctx *ctx = nullptr;
    int Nv = 0, Nt = 0, Ne = 0, patchEdge = 0, groundEdge = 0;
    DevBuf V, F, edge, ti, sg, zs, fl;   // ti: plusTri, minusTri; sg: plusSign, minusSign; fl: the doubles
};

extern "C" efie_status efie_design_build(efie_ctx *ctx, double Lp, double Wp, double Lg, double Wg, double h,
                                         int32_t Npx, int32_t Npy, int32_t Ngx, int32_t Ngy, int32_t vertex_order,
                                         const double feed[2], efie_design **out) {
    if (!ctx || !out || !feed) return efie_fail(EFIE_ERR_ARGS, "design: null argument");
    *out = nullptr;
    if (Npx < 1 || Npy < 1 || Ngx < 1 || Ngy < 1)
        return efie_fail(EFIE_ERR_ARGS, "mesh: grid sizes must be >= 1 and outputs non-null");
    if (vertex_order != 0 && vertex_order != 1) return efie_fail(EFIE_ERR_ARGS, "mesh: vertex_order must be 0 or 1");
    const long long nvp = (long long)(Npx + 1) * (Npy + 1), nvg = (long long)(Ngx + 1) * (Ngy + 1);
    const long long ntl = 2 * ((long long)Npx * Npy + (long long)Ngx * Ngy);
    if (nvp + nvg > (1 << 26) || ntl > (1 << 26)) return efie_fail(EFIE_ERR_ARGS, "design: mesh too large");
    DeviceGuard dg(ctx->device);
    efie_design *d = new (std::nothrow) efie_design();
    if (!d) return efie_fail(EFIE_ERR_NOMEM, "out of host memory");
    d->ctx = ctx;
    const int Nv = (int)(nvp + nvg), Nt = (int)ntl;
    d->Nv = Nv;
    d->Nt = Nt;
    cudaStream_t s = ctx->stream;
    auto fail = [&](efie_status st) {
        delete d;
        return st;
    };
    DevBuf cnt, off, fill, bucket, icnt, eoff, zmid, flags;
    efie_status st = EFIE_OK;
    if ((st = d->V.reserve(sizeof(double) * 3 * (size_t)Nv)) != EFIE_OK ||
        (st = d->F.reserve(sizeof(int) * 3 * (size_t)Nt)) != EFIE_OK ||
        (st = cnt.reserve(sizeof(int) * Nv)) != EFIE_OK || (st = off.reserve(sizeof(int) * (Nv + 1))) != EFIE_OK ||
        (st = fill.reserve(sizeof(int) * Nv)) != EFIE_OK || (st = bucket.reserve(sizeof(int) * 3 * (size_t)Nt)) != EFIE_OK ||
        (st = icnt.reserve(sizeof(int) * Nv)) != EFIE_OK || (st = eoff.reserve(sizeof(int) * (Nv + 1))) != EFIE_OK ||
        (st = zmid.reserve(sizeof(double))) != EFIE_OK || (st = flags.reserve(sizeof(int) * 4)) != EFIE_OK)
        return fail(st);
    const Plate P0{Wp, Lp, +h / 2, Npx, Npy, 0, 0};
    const Plate P1{Wg, Lg, -h / 2, Ngx, Ngy, (int)nvp, 2 * Npx * Npy};
    const long long most = std::max({nvp, nvg, (long long)Npx * Npy, (long long)Ngx * Ngy});
    int *fl = flags.as<int>();
    cudaError_t e = cudaMemsetAsync(flags.p, 0, sizeof(int) * 4, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(cnt.p, 0, sizeof(int) * Nv, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(fill.p, 0, sizeof(int) * Nv, s);
    if (e == cudaSuccess) {
        k_mesh<<<dim3((unsigned)((most + 255) / 256), 2), 256, 0, s>>>(P0, P1, Nv, Nt, vertex_order,
                                                                        d->V.as<double>(), d->F.as<int>());
        const int g3 = (3 * Nt + 255) / 256, gv = (Nv + 255) / 256;
        k_raw_count<<<g3, 256, 0, s>>>(Nv, Nt, d->F.as<int>(), cnt.as<int>(), fl);
        k_scan<<<1, 1024, 0, s>>>(Nv, cnt.as<int>(), off.as<int>());
        k_raw_scatter<<<g3, 256, 0, s>>>(Nv, Nt, d->F.as<int>(), off.as<int>(), fill.as<int>(), bucket.as<int>());
        k_bucket_sort<<<gv, 256, 0, s>>>(Nv, Nt, d->F.as<int>(), off.as<int>(), bucket.as<int>(), icnt.as<int>());
        k_scan<<<1, 1024, 0, s>>>(Nv, icnt.as<int>(), eoff.as<int>());
        k_zmid<<<1, 1024, 0, s>>>(Nv, d->V.as<double>(), zmid.as<double>());
        e = cudaGetLastError();
    }
    int hne = 0, hbad = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hne, eoff.as<int>() + Nv, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hbad, fl, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(efie_fail(EFIE_ERR_CUDA, std::string("design: ") + cudaGetErrorString(e)));
    if (hbad) return fail(efie_fail(EFIE_ERR_F, "rwg: F has invalid indices."));
    if (hne < 1) return fail(efie_fail(EFIE_ERR_MESH, "rwg: the mesh has no interior edge"));
    const int Ne = hne;
    d->Ne = Ne;
    if ((st = d->edge.reserve(sizeof(int) * 2 * (size_t)Ne)) != EFIE_OK ||
        (st = d->ti.reserve(sizeof(int) * 2 * (size_t)Ne)) != EFIE_OK ||
        (st = d->sg.reserve(sizeof(int) * 2 * (size_t)Ne)) != EFIE_OK ||
        (st = d->zs.reserve(sizeof(int) * (size_t)Ne)) != EFIE_OK ||
        (st = d->fl.reserve(sizeof(double) * 15 * (size_t)Ne)) != EFIE_OK)
        return fail(st);
    double *fd = d->fl.as<double>();
    RwgOut o{d->edge.as<int>(), d->ti.as<int>(), d->ti.as<int>() + Ne, d->sg.as<int>(), d->sg.as<int>() + Ne,
             d->zs.as<int>(), fd, fd + 3 * (size_t)Ne, fd + 6 * (size_t)Ne, fd + 7 * (size_t)Ne, fd + 8 * (size_t)Ne,
             fd + 9 * (size_t)Ne};
    k_rwg_fill<<<(Nv + 255) / 256, 256, 0, s>>>(Nv, Nt, Ne, d->V.as<double>(), d->F.as<int>(), off.as<int>(),
                                                 bucket.as<int>(), eoff.as<int>(), zmid.as<double>(), o, fl);
    // port edges: nearest edge centres to (feed, +h/2) on the patch layer and
    // (feed, -h/2) on the ground layer (main_patch_gpu_mex_sweep_l.m:42-43)
    k_pick_port<<<1, 1024, 0, s>>>(Ne, o.center, o.zSign, feed[0], feed[1], +h / 2, +1, fl + 1);
    k_pick_port<<<1, 1024, 0, s>>>(Ne, o.center, o.zSign, feed[0], feed[1], -h / 2, -1, fl + 2);
    e = cudaGetLastError();
    int hf[3] = {0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(hf, fl, sizeof(int) * 3, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(efie_fail(EFIE_ERR_CUDA, std::string("design: ") + cudaGetErrorString(e)));
    if (hf[0] == 2) return fail(efie_fail(EFIE_ERR_MESH, "rwg: opposite vertex not found."));
    if (hf[1] < 1 || hf[2] < 1) return fail(efie_fail(EFIE_ERR_PORT, "port: no edge on this layer"));
    d->patchEdge = hf[1];
    d->groundEdge = hf[2];
    *out = d;
    return EFIE_OK;
}

extern "C" efie_status efie_design_sizes(const efie_design *d, int32_t *Nv, int32_t *Nt, int32_t *Ne,
                                         int32_t *patchEdge, int32_t *groundEdge) {
    if (!d) return efie_fail(EFIE_ERR_ARGS, "null design");
    if (Nv) *Nv = d->Nv;
    if (Nt) *Nt = d->Nt;
    if (Ne) *Ne = d->Ne;
    if (patchEdge) *patchEdge = d->patchEdge;
    if (groundEdge) *groundEdge = d->groundEdge;
    return EFIE_OK;
}

extern "C" efie_status efie_design_read(const efie_design *d, double *V, int32_t *F, int32_t *edge, int32_t *plusTri,
                                        int32_t *minusTri, int32_t *plusSign, int32_t *minusSign, double *rp,
                                        double *rm, double *Ap, double *Am, double *len, double *center,
                                        int32_t *zSign) {
    if (!d) return efie_fail(EFIE_ERR_ARGS, "null design");
    DeviceGuard dg(d->ctx->device);
    cudaStream_t s = d->ctx->stream;
    const size_t Ne = d->Ne;
    const double *fd = d->fl.as<double>();
    auto down = [&](void *dst, const void *src, size_t bytes) -> efie_status {
        if (dst) EFIE_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
        return EFIE_OK;
    };
    EFIE_TRY(down(V, d->V.p, sizeof(double) * 3 * (size_t)d->Nv));
    EFIE_TRY(down(F, d->F.p, sizeof(int) * 3 * (size_t)d->Nt));
    EFIE_TRY(down(edge, d->edge.p, sizeof(int) * 2 * Ne));
    EFIE_TRY(down(plusTri, d->ti.as<int>(), sizeof(int) * Ne));
    EFIE_TRY(down(minusTri, d->ti.as<int>() + Ne, sizeof(int) * Ne));
    EFIE_TRY(down(plusSign, d->sg.as<int>(), sizeof(int) * Ne));
    EFIE_TRY(down(minusSign, d->sg.as<int>() + Ne, sizeof(int) * Ne));
    EFIE_TRY(down(rp, fd, sizeof(double) * 3 * Ne));
    EFIE_TRY(down(rm, fd + 3 * Ne, sizeof(double) * 3 * Ne));
    EFIE_TRY(down(Ap, fd + 6 * Ne, sizeof(double) * Ne));
    EFIE_TRY(down(Am, fd + 7 * Ne, sizeof(double) * Ne));
    EFIE_TRY(down(len, fd + 8 * Ne, sizeof(double) * Ne));
    EFIE_TRY(down(center, fd + 9 * Ne, sizeof(double) * 3 * Ne));
    EFIE_TRY(down(zSign, d->zs.p, sizeof(int) * Ne));
    EFIE_CUDA(cudaStreamSynchronize(s));
    return EFIE_OK;
}

extern "C" void efie_design_destroy(efie_design *d) {
    if (!d) return;
    DeviceGuard dg(d->ctx->device);
    cudaStreamSynchronize(d->ctx->stream);
    delete d;
}
