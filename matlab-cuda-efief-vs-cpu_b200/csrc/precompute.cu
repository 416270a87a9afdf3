// efie_precompute + efie_precompute_pack on the GPU (efie_precompute.m:1-97,
// efie_precompute_pack.m:1-59): per-triangle quadrature caches (regular rule,
// self- and near-subdivided rules, softening lengths) and the near-pair
// relation, computed from V and F on the device.
//
// The reference (and efie_precompute_pack in geom.cpp) builds an Nt x Nt uint8
// nearMat on the host and hands it to the MEX (22 MB at Ne 6968, 180 MB at Ne
// 19936), which then has to be scanned for the near pairs.  Here the relation
// D(t1,t2) < eps/2 (h1 + h2) is evaluated on the device and compacted straight
// into the ordered near-pair list the assembly uses (t2 ascending, then t1):
// the Nt^2 bytes are never formed for a plan.  efie_precompute_pack_gpu also
// writes the reference's packed arrays, nearMat included, for callers that
// want them.
//
// Every floating-point operation is an explicitly rounded IEEE operation in
// the reference's order (no contraction into FMA), so the outputs are
// bit-identical to the host producers and to the numpy restatement: the
// integer relation can then not differ on a borderline pair.
#include <algorithm>
#include <cmath>
#include <vector>

#include "efie_internal.h"

namespace {

constexpr double kPi = 3.141592653589793238462643383279502884;   // M_PI

struct Rule {
    int n;
    double u[7], v[7], w[7];
};

struct P3 {
    double x, y, z;
};

__device__ __forceinline__ double ad(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sb(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ml(double a, double b) { return __dmul_rn(a, b); }

__device__ __forceinline__ P3 vertex(const double *V, int Nv, int id1) {
    const int i = id1 - 1;
    return P3{V[i], V[i + Nv], V[i + 2 * (size_t)Nv]};
}

// |(b - a) x (c - a)| = 2A (precompute_tri_geom.m:16)
__device__ __forceinline__ double area2_of(P3 a, P3 b, P3 c) {
    const double e1x = sb(b.x, a.x), e1y = sb(b.y, a.y), e1z = sb(b.z, a.z);
    const double e2x = sb(c.x, a.x), e2y = sb(c.y, a.y), e2z = sb(c.z, a.z);
    const double cx = sb(ml(e1y, e2z), ml(e1z, e2y));
    const double cy = sb(ml(e1z, e2x), ml(e1x, e2z));
    const double cz = sb(ml(e1x, e2y), ml(e1y, e2x));
    return __dsqrt_rn(ad(ad(ml(cx, cx), ml(cy, cy)), ml(cz, cz)));
}

// map_ref_to_vertices.m: r = A + u (B - A) + v (C - A)
__device__ __forceinline__ P3 map_point(P3 A, P3 B, P3 C, double u, double v) {
    return P3{ad(ad(A.x, ml(u, sb(B.x, A.x))), ml(v, sb(C.x, A.x))),
              ad(ad(A.y, ml(u, sb(B.y, A.y))), ml(v, sb(C.y, A.y))),
              ad(ad(A.z, ml(u, sb(B.z, A.z))), ml(v, sb(C.z, A.z)))};
}

__device__ __forceinline__ P3 mid(P3 a, P3 b) { return P3{ml(0.5, ad(a.x, b.x)), ml(0.5, ad(a.y, b.y)), ml(0.5, ad(a.z, b.z))}; }

// Sub-triangle p of `depth` midpoint subdivisions (subdivide_triangles.m:1-20):
// each level appends the children A-AB-CA, AB-B-BC, CA-BC-C, AB-BC-CA of every
// triangle in order, so the base-4 digits of p, most significant first, pick
// the child at each level.
__device__ __forceinline__ void sub_triangle(P3 &A, P3 &B, P3 &C, int depth, int p) {
    for (int l = 0; l < depth; l++) {
        const int k = (p >> (2 * (depth - 1 - l))) & 3;
        const P3 AB = mid(A, B), BC = mid(B, C), CA = mid(C, A);
        if (k == 0) B = AB, C = CA;
        else if (k == 1) A = AB, C = BC;
        else if (k == 2) A = CA, B = BC;
        else A = AB, B = BC, C = CA;
    }
}

struct PackOut {          // the reference's packed arrays (column-major), or null
    double *r_reg, *w_reg, *self_r, *self_w, *self_a, *near_r, *near_w, *aeq;
};

struct PlanOut {          // the assembly's layout: points relative to the centroid, weight in w
    double4 *origin, *reg, *nearp, *selfp;
    double *self_a, *aeq;
};

// Thread (t, p): sub-triangle p of the self and near subdivisions of triangle
// t; p == 0 also writes the triangle's centroid, h, aeqTri and regular points.
template <bool PLAN>
__global__ void __launch_bounds__(128) k_pre_triangles(int Nv, int Nt, const double *__restrict__ V,
                                                       const int *__restrict__ F, Rule reg, Rule sub, int dS, int dN,
                                                       double self_alpha, PackOut po, PlanOut pl,
                                                       double4 *__restrict__ cent_h, int *__restrict__ bad) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int p = blockIdx.y;
    if (t >= Nt) return;
    const int i1 = F[t], i2 = F[t + Nt], i3 = F[t + 2 * (size_t)Nt];
    if (i1 < 1 || i1 > Nv || i2 < 1 || i2 > Nv || i3 < 1 || i3 > Nv) {
        if (p == 0) atomicExch(bad, 1);
        return;
    }
    const P3 r1 = vertex(V, Nv, i1), r2 = vertex(V, Nv, i2), r3 = vertex(V, Nv, i3);
    // centroid (precompute_tri_geom.m:15), the origin of the plan's local coordinates
    const P3 o{__ddiv_rn(ad(ad(r1.x, r2.x), r3.x), 3.0), __ddiv_rn(ad(ad(r1.y, r2.y), r3.y), 3.0),
               __ddiv_rn(ad(ad(r1.z, r2.z), r3.z), 3.0)};
    const int NsS = 1 << (2 * dS), NsN = 1 << (2 * dN);
    if (p == 0) {
        const double a2 = area2_of(r1, r2, r3);
        const double h = __dsqrt_rn(__ddiv_rn(ml(2.0, a2), __dsqrt_rn(3.0)));   // efie_precompute.m:19
        const double aeq = __dsqrt_rn(__ddiv_rn(ml(0.5, a2), kPi));            // :41-42
        cent_h[t] = make_double4(o.x, o.y, o.z, h);
        for (int i = 0; i < reg.n; i++) {                                       // :32-38
            const P3 r = map_point(r1, r2, r3, reg.u[i], reg.v[i]);
            const double w = ml(reg.w[i], a2);
            if (PLAN) {
                pl.reg[(size_t)t * reg.n + i] = make_double4(sb(r.x, o.x), sb(r.y, o.y), sb(r.z, o.z), w);
            } else {
                double *R = po.r_reg + i + (size_t)reg.n * 3 * t;
                R[0] = r.x;
                R[reg.n] = r.y;
                R[2 * reg.n] = r.z;
                po.w_reg[i + (size_t)reg.n * t] = w;
            }
        }
        if (PLAN) {
            pl.origin[t] = make_double4(o.x, o.y, o.z, 0.0);
            pl.aeq[t] = aeq;
        } else {
            po.aeq[t] = aeq;
        }
    }
    for (int pass = 0; pass < 2; pass++) {                                      // :52-95
        const bool self = pass == 0;
        const int Ns = self ? NsS : NsN;
        if (p >= Ns) continue;
        P3 A = r1, B = r2, C = r3;
        sub_triangle(A, B, C, self ? dS : dN, p);
        const double a2p = area2_of(A, B, C);                                   // :67 / :88
        for (int i = 0; i < sub.n; i++) {
            const P3 r = map_point(A, B, C, sub.u[i], sub.v[i]);
            const double w = ml(sub.w[i], a2p);
            if (PLAN) {
                double4 *dst = self ? pl.selfp : pl.nearp;
                dst[((size_t)t * Ns + p) * sub.n + i] = make_double4(sb(r.x, o.x), sb(r.y, o.y), sb(r.z, o.z), w);
            } else {
                double *R = (self ? po.self_r : po.near_r) + i + (size_t)sub.n * 3 * p + (size_t)sub.n * 3 * Ns * t;
                R[0] = r.x;
                R[sub.n] = r.y;
                R[2 * sub.n] = r.z;
                (self ? po.self_w : po.near_w)[i + (size_t)sub.n * p + (size_t)sub.n * Ns * t] = w;
            }
        }
        if (self) {
            const double a = ml(self_alpha, __dsqrt_rn(__ddiv_rn(ml(0.5, a2p), kPi)));   // :71-73
            (PLAN ? pl.self_a : po.self_a)[p + (size_t)NsS * t] = a;
        }
    }
}

// nearMat(t1,t2) = D < eps/2 (h1 + h2), D the centroid distance (efie_precompute.m:24-29)
__device__ __forceinline__ bool is_near(const double4 &a, const double4 &b, double eps) {
    const double dx = sb(a.x, b.x), dy = sb(a.y, b.y), dz = sb(a.z, b.z);
    const double D = __dsqrt_rn(ad(ad(ml(dx, dx), ml(dy, dy)), ml(dz, dz)));
    return D < ml(ml(eps, 0.5), ad(a.w, b.w));
}

// The whole relation, column-major uint8 (the reference's nearMat).
__global__ void __launch_bounds__(256) k_near_mat(int Nt, const double4 *__restrict__ ch, double eps,
                                                  uint8_t *__restrict__ nm) {
    const int t1 = blockIdx.x * blockDim.x + threadIdx.x, t2 = blockIdx.y;
    if (t1 >= Nt) return;
    nm[(size_t)t1 + (size_t)Nt * t2] = is_near(ch[t1], ch[t2], eps) ? 1 : 0;
}

// Near pairs t1 < t2 of column t2 (one CTA per column): the count, or (with
// `list`) the pairs themselves, in increasing t1 from offset[t2] on.  The
// relation is symmetric bit for bit (the same rounded operations on exactly
// negated differences), so the upper triangle carries all of it.
__global__ void __launch_bounds__(256) k_near_pairs(int Nt, const double4 *__restrict__ ch, double eps,
                                                    int *__restrict__ count, const long long *__restrict__ offset,
                                                    int2 *__restrict__ list) {
    __shared__ int warp_n[8];
    __shared__ long long base_sh;
    const int t2 = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const double4 c2 = ch[t2];
    if (tid == 0) base_sh = list ? offset[t2] : 0;
    __syncthreads();
    int total = 0;
    for (int c0 = 0; c0 < t2; c0 += 256) {
        const int t1 = c0 + tid;
        const bool nr = t1 < t2 && is_near(ch[t1], c2, eps);
        const unsigned bal = __ballot_sync(0xffffffffu, nr);
        if (lane == 0) warp_n[warp] = __popc(bal);
        __syncthreads();
        int before = 0, chunk = 0;
        for (int w = 0; w < 8; w++) {
            if (w < warp) before += warp_n[w];
            chunk += warp_n[w];
        }
        if (list && nr) list[base_sh + total + before + __popc(bal & ((1u << lane) - 1u))] = make_int2(t1, t2);
        total += chunk;
        __syncthreads();
    }
    if (!list && tid == 0) count[t2] = total;
}

// Exclusive prefix sum of the per-column counts (one CTA); offset[Nt] = total.
__global__ void __launch_bounds__(1024) k_scan_counts(int Nt, const int *__restrict__ count,
                                                      long long *__restrict__ offset) {
    __shared__ long long part[1024];
    const int tid = threadIdx.x;
    const int per = (Nt + 1023) / 1024;
    const int b0 = min(Nt, tid * per), b1 = min(Nt, b0 + per);
    long long s = 0;
    for (int i = b0; i < b1; i++) s += count[i];
    part[tid] = s;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const long long v = tid >= o ? part[tid - o] : 0;
        __syncthreads();
        part[tid] += v;
        __syncthreads();
    }
    long long run = tid ? part[tid - 1] : 0;
    for (int i = b0; i < b1; i++) {
        offset[i] = run;
        run += count[i];
    }
    if (tid == 1023) offset[Nt] = part[1023];
}

efie_status rules_of(const efie_precompute_opts *o, Rule &reg, Rule &sub) {
    if (o->self_subdiv < 0 || o->self_subdiv > 6 || o->near_subdiv < 0 || o->near_subdiv > 6)
        return efie_fail(EFIE_ERR_ARGS, "precompute: subdivision depth must be in [0, 6]");
    reg.n = efie_quad_rule(o->quad_order, reg.u, reg.v, reg.w);
    sub.n = efie_quad_rule(o->near_order, sub.u, sub.v, sub.w);
    return EFIE_OK;
}

// V and F on the device plus the per-triangle kernels; cent_h receives the
// centroids and h of every triangle.
template <bool PLAN>
efie_status run_triangles(efie_ctx *ctx, int Nv, const double *V, int Nt, const int *F,
                          const efie_precompute_opts *o, const PackOut &po, const PlanOut &pl, DevBuf &cent_h) {
    Rule reg, sub;
    EFIE_TRY(rules_of(o, reg, sub));
    cudaStream_t s = ctx->stream;
    DevBuf dV, dF, bad;
    EFIE_TRY(dV.reserve(sizeof(double) * 3 * (size_t)Nv));
    EFIE_TRY(dF.reserve(sizeof(int) * 3 * (size_t)Nt));
    EFIE_TRY(bad.reserve(sizeof(int)));
    EFIE_TRY(cent_h.reserve(sizeof(double4) * Nt));
    EFIE_CUDA(cudaMemcpyAsync(dV.p, V, sizeof(double) * 3 * (size_t)Nv, cudaMemcpyHostToDevice, s));
    EFIE_CUDA(cudaMemcpyAsync(dF.p, F, sizeof(int) * 3 * (size_t)Nt, cudaMemcpyHostToDevice, s));
    EFIE_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), s));
    const int ns = std::max(1 << (2 * o->self_subdiv), 1 << (2 * o->near_subdiv));
    k_pre_triangles<PLAN><<<dim3((Nt + 127) / 128, ns), 128, 0, s>>>(
        Nv, Nt, dV.as<double>(), dF.as<int>(), reg, sub, o->self_subdiv, o->near_subdiv, o->self_alpha, po, pl,
        cent_h.as<double4>(), bad.as<int>());
    EFIE_CUDA(cudaGetLastError());
    int hbad = 0;
    EFIE_CUDA(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    EFIE_CUDA(cudaStreamSynchronize(s));
    if (hbad) return efie_fail(EFIE_ERR_F, "precompute: F has invalid indices.");
    return EFIE_OK;
}

}  // namespace

// Plan geometry of the reference scheme from V/F on the device (efie_geom_upload
// with no host prepack): the caches in the assembly's layout and the ordered
// near-pair list.  g.origin must not be set yet; it is written here.
efie_status efie_geom_precompute_device(efie_ctx *ctx, const efie_mesh *mesh, const efie_precompute_opts *o,
                                        GeomDev &g) {
    const int Nt = mesh->Nt;
    Rule reg, sub;
    EFIE_TRY(rules_of(o, reg, sub));
    g.Nq = reg.n;
    g.Nq2 = sub.n;
    g.NsS = 1 << (2 * o->self_subdiv);
    g.NsN = 1 << (2 * o->near_subdiv);
    g.near_alpha = o->near_alpha;
    EFIE_TRY(g.origin.reserve(sizeof(double4) * Nt));
    EFIE_TRY(g.reg_pts.reserve(sizeof(double4) * (size_t)Nt * g.Nq));
    EFIE_TRY(g.near_pts.reserve(sizeof(double4) * (size_t)Nt * g.NsN * g.Nq2));
    EFIE_TRY(g.self_pts.reserve(sizeof(double4) * (size_t)Nt * g.NsS * g.Nq2));
    EFIE_TRY(g.self_a.reserve(sizeof(double) * (size_t)Nt * g.NsS));
    EFIE_TRY(g.aeq.reserve(sizeof(double) * Nt));
    PlanOut pl{g.origin.as<double4>(), g.reg_pts.as<double4>(), g.near_pts.as<double4>(), g.self_pts.as<double4>(),
               g.self_a.as<double>(), g.aeq.as<double>()};
    DevBuf ch;
    EFIE_TRY(run_triangles<true>(ctx, mesh->Nv, mesh->V, Nt, mesh->F, o, PackOut{}, pl, ch));
    // near pairs: count per column, offsets, ordered fill
    cudaStream_t s = ctx->stream;
    DevBuf cnt, off;
    EFIE_TRY(cnt.reserve(sizeof(int) * Nt));
    EFIE_TRY(off.reserve(sizeof(long long) * (Nt + 1)));
    k_near_pairs<<<Nt, 256, 0, s>>>(Nt, ch.as<double4>(), o->near_sing_eps, cnt.as<int>(), nullptr, nullptr);
    k_scan_counts<<<1, 1024, 0, s>>>(Nt, cnt.as<int>(), off.as<long long>());
    EFIE_CUDA(cudaGetLastError());
    long long total = 0;
    EFIE_CUDA(cudaMemcpyAsync(&total, off.as<long long>() + Nt, sizeof(long long), cudaMemcpyDeviceToHost, s));
    EFIE_CUDA(cudaStreamSynchronize(s));
    if (total > (long long)INT32_MAX) return efie_fail(EFIE_ERR_ARGS, "precompute: too many near pairs");
    EFIE_TRY(g.near_list.reserve(sizeof(int2) * std::max<long long>(total, 1)));
    if (total > 0)
        k_near_pairs<<<Nt, 256, 0, s>>>(Nt, ch.as<double4>(), o->near_sing_eps, nullptr, off.as<long long>(),
                                        g.near_list.as<int2>());
    EFIE_CUDA(cudaGetLastError());
    g.n_near = (int)total;
    g.symmetric = true;
    EFIE_CUDA(cudaStreamSynchronize(s));   // the temporaries go back to the pool after this
    return EFIE_OK;
}

extern "C" efie_status efie_precompute_pack_gpu(efie_ctx *ctx, int32_t Nv, const double *V, int32_t Nt,
                                                const int32_t *F, const efie_precompute_opts *o, efie_prepack *out) {
    if (!ctx || !V || !F || !o || !out || Nt < 1 || Nv < 1)
        return efie_fail(EFIE_ERR_ARGS, "precompute: bad arguments");
    const int Nq = efie_quad_rule_size(o->quad_order), Nq2 = efie_quad_rule_size(o->near_order);
    if (o->self_subdiv < 0 || o->self_subdiv > 6 || o->near_subdiv < 0 || o->near_subdiv > 6)
        return efie_fail(EFIE_ERR_ARGS, "precompute: subdivision depth must be in [0, 6]");
    const int NsS = 1 << (2 * o->self_subdiv), NsN = 1 << (2 * o->near_subdiv);
    if (out->Nt != Nt || out->Nq != Nq || out->Nq2 != Nq2 || out->NsS != NsS || out->NsN != NsN)
        return efie_fail(EFIE_ERR_PREPACK, "precompute: output dimensions do not match the options");
    if (!out->r_reg || !out->w_reg || !out->nearMat || !out->self_r || !out->self_w || !out->self_a ||
        !out->near_r || !out->near_w || !out->aeqTri)
        return efie_fail(EFIE_ERR_PREPACK, "precompute: null output array");
    if (Nt > 65535) return efie_fail(EFIE_ERR_ARGS, "precompute: nearMat output limited to Nt <= 65535");
    DeviceGuard dg(ctx->device);
    const size_t n_reg = (size_t)Nq * Nt, n_self = (size_t)Nq2 * NsS * Nt, n_near = (size_t)Nq2 * NsN * Nt;
    const size_t nd = 4 * n_reg + 4 * n_self + (size_t)NsS * Nt + 4 * n_near + Nt;   // doubles of the packed arrays
    DevBuf buf, nm, ch;
    EFIE_TRY(buf.reserve(sizeof(double) * nd));
    EFIE_TRY(nm.reserve((size_t)Nt * Nt));
    double *d = buf.as<double>();
    PackOut po;
    po.r_reg = d;  d += 3 * n_reg;
    po.w_reg = d;  d += n_reg;
    po.self_r = d; d += 3 * n_self;
    po.self_w = d; d += n_self;
    po.self_a = d; d += (size_t)NsS * Nt;
    po.near_r = d; d += 3 * n_near;
    po.near_w = d; d += n_near;
    po.aeq = d;
    EFIE_TRY(run_triangles<false>(ctx, Nv, V, Nt, F, o, po, PlanOut{}, ch));
    cudaStream_t s = ctx->stream;
    k_near_mat<<<dim3((Nt + 255) / 256, Nt), 256, 0, s>>>(Nt, ch.as<double4>(), o->near_sing_eps, nm.as<uint8_t>());
    EFIE_CUDA(cudaGetLastError());
    auto down = [&](void *dst, const void *src, size_t bytes) -> efie_status {
        EFIE_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
        return EFIE_OK;
    };
    EFIE_TRY(down(out->r_reg, po.r_reg, sizeof(double) * 3 * n_reg));
    EFIE_TRY(down(out->w_reg, po.w_reg, sizeof(double) * n_reg));
    EFIE_TRY(down(out->self_r, po.self_r, sizeof(double) * 3 * n_self));
    EFIE_TRY(down(out->self_w, po.self_w, sizeof(double) * n_self));
    EFIE_TRY(down(out->self_a, po.self_a, sizeof(double) * NsS * (size_t)Nt));
    EFIE_TRY(down(out->near_r, po.near_r, sizeof(double) * 3 * n_near));
    EFIE_TRY(down(out->near_w, po.near_w, sizeof(double) * n_near));
    EFIE_TRY(down(out->aeqTri, po.aeq, sizeof(double) * Nt));
    EFIE_TRY(down(out->nearMat, nm.p, (size_t)Nt * Nt));
    EFIE_CUDA(cudaStreamSynchronize(s));
    out->near_alpha = o->near_alpha;
    out->self_alpha = o->self_alpha;
    return EFIE_OK;
}
