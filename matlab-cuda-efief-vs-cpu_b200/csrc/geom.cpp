// Host-side producers of the MEX boundary data: mesh, RWG topology, port
// edges, quadrature rules and the efie_precompute_pack cache.  In the
// reference these run in MATLAB before the MEX call; here they are native so
// that design families can be generated without MATLAB.  Index outputs are
// 1-based int32 and arrays are column-major, exactly as MATLAB produces them.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "efie_internal.h"

namespace {

// MATLAB linspace: d1 + (0:n1).*(d2-d1)./n1, ends pinned (multiply first,
// then divide).
void linspace_matlab(double d1, double d2, int n, std::vector<double> &y) {
    y.resize(n);
    int n1 = n - 1;
    for (int i = 0; i < n; i++) y[i] = d1 + ((double)i * (d2 - d1)) / (double)n1;
    y[0] = d1;
    y[n - 1] = d2;
}

inline double norm3(double x, double y, double z) { return std::sqrt(x * x + y * y + z * z); }

inline double area2_of(const double *r1, const double *r2, const double *r3) {
    double e1[3] = {r2[0] - r1[0], r2[1] - r1[1], r2[2] - r1[2]};
    double e2[3] = {r3[0] - r1[0], r3[1] - r1[1], r3[2] - r1[2]};
    double cx = e1[1] * e2[2] - e1[2] * e2[1];
    double cy = e1[2] * e2[0] - e1[0] * e2[2];
    double cz = e1[0] * e2[1] - e1[1] * e2[0];
    return norm3(cx, cy, cz);
}

}  // namespace

extern "C" int32_t efie_quad_rule_size(int32_t order) {
    if (order == EFIE_QUAD_DUNAVANT7) return 7;
    if (order == 1) return 1;
    if (order == 2) return 3;
    return 6;
}

// tri_quad_rule.m:1-23 (reference triangle (0,0),(1,0),(0,1), weights sum 1/2)
// plus the Dunavant (1985) degree-5 7-point rule.
int efie_quad_rule(int order, double *u, double *v, double *w) {
    if (order == EFIE_QUAD_DUNAVANT7) {
        const double s15 = std::sqrt(15.0);
        const double a1 = (6.0 - s15) / 21.0, a2 = (6.0 + s15) / 21.0;
        const double w0 = 9.0 / 40.0, w1 = (155.0 - s15) / 1200.0, w2 = (155.0 + s15) / 1200.0;
        const double uu[7] = {1.0 / 3.0, a1, 1 - 2 * a1, a1, a2, 1 - 2 * a2, a2};
        const double vv[7] = {1.0 / 3.0, a1, a1, 1 - 2 * a1, a2, a2, 1 - 2 * a2};
        const double ww[7] = {w0, w1, w1, w1, w2, w2, w2};
        for (int i = 0; i < 7; i++) { u[i] = uu[i]; v[i] = vv[i]; w[i] = 0.5 * ww[i]; }
        return 7;
    }
    if (order == 1) { u[0] = 1.0 / 3.0; v[0] = 1.0 / 3.0; w[0] = 0.5; return 1; }
    if (order == 2) {
        const double uu[3] = {1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0};
        const double vv[3] = {1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0};
        for (int i = 0; i < 3; i++) { u[i] = uu[i]; v[i] = vv[i]; w[i] = 1.0 / 6.0; }
        return 3;
    }
    const double a = 0.445948490915965, b = 0.108103018168070;
    const double w1 = 0.111690794839005, w2 = 0.054975871827661;
    const double uu[6] = {a, a, 1 - 2 * a, b, b, 1 - 2 * b};
    const double vv[6] = {a, 1 - 2 * a, a, b, 1 - 2 * b, b};
    const double ww[6] = {w1, w1, w1, w2, w2, w2};
    for (int i = 0; i < 6; i++) { u[i] = uu[i]; v[i] = vv[i]; w[i] = ww[i]; }
    return 6;
}

extern "C" efie_status efie_make_patch_with_ground_mesh(double Lp, double Wp, double Lg, double Wg, double h,
                                                        int32_t Npx, int32_t Npy, int32_t Ngx, int32_t Ngy,
                                                        int32_t vertex_order, double *V, int32_t *F) {
    if (Npx < 1 || Npy < 1 || Ngx < 1 || Ngy < 1 || !V || !F)
        return efie_fail(EFIE_ERR_ARGS, "mesh: grid sizes must be >= 1 and outputs non-null");
    if (vertex_order != 0 && vertex_order != 1) return efie_fail(EFIE_ERR_ARGS, "mesh: vertex_order must be 0 or 1");
    const int64_t Nvp = (int64_t)(Npx + 1) * (Npy + 1), Nvg = (int64_t)(Ngx + 1) * (Ngy + 1);
    const int64_t Nv = Nvp + Nvg;
    const int64_t Nt = 2 * ((int64_t)Npx * Npy + (int64_t)Ngx * Ngy);
    struct Plate { double W, L, z; int nx, ny; int64_t voff, toff; };
    Plate plates[2] = {{Wp, Lp, +h / 2, Npx, Npy, 0, 0},
                       {Wg, Lg, -h / 2, Ngx, Ngy, Nvp, 2 * (int64_t)Npx * Npy}};
    std::vector<double> xs, ys;
    for (const Plate &P : plates) {
        // make_patch_with_ground_mesh.m:5-7 / :23-25
        linspace_matlab(-P.W / 2, P.W / 2, P.nx + 1, xs);
        linspace_matlab(-P.L / 2, P.L / 2, P.ny + 1, ys);
        for (int i = 0; i <= P.nx; i++)
            for (int j = 0; j <= P.ny; j++) {
                // reference: meshgrid(:) is column-major, y fastest
                int64_t local = vertex_order == 0 ? (int64_t)j + (int64_t)i * (P.ny + 1)
                                                  : (int64_t)i + (int64_t)j * (P.nx + 1);
                int64_t vi = P.voff + local;
                V[vi] = xs[i];
                V[vi + Nv] = ys[j];
                V[vi + 2 * Nv] = P.z;
            }
        // :9-20 / :27-39 faces, x-fastest indexing
        int64_t t = P.toff;
        for (int j = 1; j <= P.ny; j++)
            for (int i = 1; i <= P.nx; i++) {
                int64_t v1 = P.voff + (int64_t)(j - 1) * (P.nx + 1) + i;
                int64_t v2 = v1 + 1, v3 = v1 + (P.nx + 1), v4 = v3 + 1;
                F[t] = (int32_t)v1; F[t + Nt] = (int32_t)v2; F[t + 2 * Nt] = (int32_t)v4; t++;
                F[t] = (int32_t)v1; F[t + Nt] = (int32_t)v4; F[t + 2 * Nt] = (int32_t)v3; t++;
            }
    }
    return EFIE_OK;
}

extern "C" efie_status efie_build_rwg_interior(int32_t Nv, const double *V, int32_t Nt, const int32_t *F,
                                               int32_t capacity, int32_t *NeOut,
                                               int32_t *edge, int32_t *plusTri, int32_t *minusTri,
                                               int32_t *plusSign, int32_t *minusSign,
                                               double *rp, double *rm, double *Ap, double *Am,
                                               double *len, double *center, int32_t *zSign) {
    if (Nv < 1 || Nt < 1 || !V || !F || !NeOut) return efie_fail(EFIE_ERR_ARGS, "rwg: empty mesh");
    for (int64_t i = 0; i < 3 * (int64_t)Nt; i++)
        if (F[i] < 1 || F[i] > Nv) return efie_fail(EFIE_ERR_F, "rwg: F has invalid indices.");
    // build_rwg_interior.m:10-23: raw directed edges, row p = 3t + le
    struct Raw { int32_t lo, hi, a, b, tri; int32_t row; };
    std::vector<Raw> raw((size_t)Nt * 3);
    for (int32_t t = 0; t < Nt; t++) {
        int32_t v[3] = {F[t], F[t + Nt], F[t + 2 * (int64_t)Nt]};
        for (int le = 0; le < 3; le++) {
            int32_t a = v[le], b = v[(le + 1) % 3];
            Raw &r = raw[(size_t)3 * t + le];
            r.a = a; r.b = b; r.lo = std::min(a, b); r.hi = std::max(a, b); r.tri = t + 1;
            r.row = 3 * t + le;
        }
    }
    // :25 unique(...,'rows'): lexicographic order; stable sort keeps the raw
    // order inside a group, so the first member is the first incidence (:47).
    std::stable_sort(raw.begin(), raw.end(), [](const Raw &x, const Raw &y) {
        return x.lo != y.lo ? x.lo < y.lo : x.hi < y.hi;
    });
    std::vector<std::pair<size_t, size_t>> interior;  // (first, second) raw positions
    for (size_t s = 0; s < raw.size();) {
        size_t e = s + 1;
        while (e < raw.size() && raw[e].lo == raw[s].lo && raw[e].hi == raw[s].hi) e++;
        if (e - s == 2) interior.emplace_back(s, s + 1);  // :29-30 counts == 2
        s = e;
    }
    const int32_t Ne = (int32_t)interior.size();
    *NeOut = Ne;
    if (capacity == 0) return EFIE_OK;
    if (capacity != Ne) return efie_fail(EFIE_ERR_ARGS, "rwg: capacity must equal Ne");
    double zmin = V[2 * (int64_t)Nv], zmax = V[2 * (int64_t)Nv];
    for (int32_t i = 0; i < Nv; i++) {
        zmin = std::min(zmin, V[i + 2 * (int64_t)Nv]);
        zmax = std::max(zmax, V[i + 2 * (int64_t)Nv]);
    }
    const double zmid = 0.5 * (zmax + zmin);  // :88
    auto vtx = [&](int32_t id, double *r) {
        r[0] = V[id - 1]; r[1] = V[id - 1 + (int64_t)Nv]; r[2] = V[id - 1 + 2 * (int64_t)Nv];
    };
    for (int32_t e = 0; e < Ne; e++) {
        const Raw &r1 = raw[interior[e].first], &r2 = raw[interior[e].second];
        const int32_t a = r1.lo, b = r1.hi;
        // :50-63 signs relative to the (a<b) orientation
        const int32_t s1 = (r1.a == a && r1.b == b) ? 1 : -1;
        const int32_t s2 = (r2.a == a && r2.b == b) ? 1 : -1;
        if (edge) { edge[e] = a; edge[e + Ne] = b; }
        if (plusTri) plusTri[e] = r1.tri;
        if (minusTri) minusTri[e] = r2.tri;
        if (plusSign) plusSign[e] = s1;
        if (minusSign) minusSign[e] = s2;
        double ra[3], rb[3];
        vtx(a, ra);
        vtx(b, rb);
        if (len) len[e] = norm3(rb[0] - ra[0], rb[1] - ra[1], rb[2] - ra[2]);  // :75
        double c[3] = {0.5 * (ra[0] + rb[0]), 0.5 * (ra[1] + rb[1]), 0.5 * (ra[2] + rb[2])};
        if (center) for (int k = 0; k < 3; k++) center[e + (int64_t)k * Ne] = c[k];
        if (zSign) zSign[e] = c[2] > zmid ? 1 : -1;  // :89-90
        // :80-84 opposite vertex and area of the plus / minus triangle
        for (int side = 0; side < 2; side++) {
            int32_t t = side == 0 ? r1.tri : r2.tri;
            int32_t tv[3] = {F[t - 1], F[t - 1 + Nt], F[t - 1 + 2 * (int64_t)Nt]};
            int32_t opp = 0, nopp = 0;
            for (int k = 0; k < 3; k++)
                if (tv[k] != a && tv[k] != b) { opp = tv[k]; nopp++; }
            if (nopp != 1) return efie_fail(EFIE_ERR_MESH, "rwg: opposite vertex not found.");
            double p1[3], p2[3], p3[3], ro[3];
            vtx(tv[0], p1);
            vtx(tv[1], p2);
            vtx(tv[2], p3);
            vtx(opp, ro);
            double A = 0.5 * area2_of(p1, p2, p3);  // :111-112
            double *dst = side == 0 ? rp : rm;
            if (dst) for (int k = 0; k < 3; k++) dst[e + (int64_t)k * Ne] = ro[k];
            double *Ad = side == 0 ? Ap : Am;
            if (Ad) Ad[e] = A;
        }
    }
    return EFIE_OK;
}

extern "C" efie_status efie_pick_port_edge(int32_t Ne, const double *center, const int32_t *zSign,
                                           const double p[3], int32_t layerSign, int32_t *eidx) {
    if (Ne < 1 || !center || !zSign || !p || !eidx) return efie_fail(EFIE_ERR_ARGS, "port: bad arguments");
    // pick_port_edge_by_point_and_layer.m:2-10, min() keeps the first minimum
    int32_t best = -1;
    double bestd = 0.0;
    for (int32_t e = 0; e < Ne; e++) {
        if (zSign[e] != layerSign) continue;
        double dx = center[e] - p[0], dy = center[e + Ne] - p[1], dz = center[e + 2 * (int64_t)Ne] - p[2];
        double d = std::sqrt(dx * dx + dy * dy + dz * dz);
        if (best < 0 || d < bestd) { best = e; bestd = d; }
    }
    if (best < 0) return efie_fail(EFIE_ERR_PORT, "port: no edge on this layer");
    *eidx = best + 1;
    return EFIE_OK;
}

extern "C" efie_status efie_precompute_pack(int32_t Nv, const double *V, int32_t Nt, const int32_t *F,
                                            const efie_precompute_opts *o, efie_prepack *out) {
    if (!V || !F || !o || !out || Nt < 1 || Nv < 1) return efie_fail(EFIE_ERR_ARGS, "precompute: bad arguments");
    const int Nq = efie_quad_rule_size(o->quad_order), Nq2 = efie_quad_rule_size(o->near_order);
    if (o->self_subdiv < 0 || o->self_subdiv > 6 || o->near_subdiv < 0 || o->near_subdiv > 6)
        return efie_fail(EFIE_ERR_ARGS, "precompute: subdivision depth must be in [0, 6]");
    const int NsS = 1 << (2 * o->self_subdiv), NsN = 1 << (2 * o->near_subdiv);
    if (out->Nt != Nt || out->Nq != Nq || out->Nq2 != Nq2 || out->NsS != NsS || out->NsN != NsN)
        return efie_fail(EFIE_ERR_PREPACK, "precompute: output dimensions do not match the options");
    if (!out->r_reg || !out->w_reg || !out->nearMat || !out->self_r || !out->self_w || !out->self_a ||
        !out->near_r || !out->near_w || !out->aeqTri)
        return efie_fail(EFIE_ERR_PREPACK, "precompute: null output array");
    for (int64_t i = 0; i < 3 * (int64_t)Nt; i++)
        if (F[i] < 1 || F[i] > Nv) return efie_fail(EFIE_ERR_F, "precompute: F has invalid indices.");
    double qu[7], qv[7], qw[7], qu2[7], qv2[7], qw2[7];
    efie_quad_rule(o->quad_order, qu, qv, qw);
    efie_quad_rule(o->near_order, qu2, qv2, qw2);
    std::vector<double> r1(3 * (size_t)Nt), r2(3 * (size_t)Nt), r3(3 * (size_t)Nt), cent(3 * (size_t)Nt),
        area2(Nt), htri(Nt);
    for (int32_t t = 0; t < Nt; t++) {
        for (int k = 0; k < 3; k++) {
            r1[3 * t + k] = V[F[t] - 1 + (int64_t)k * Nv];
            r2[3 * t + k] = V[F[t + Nt] - 1 + (int64_t)k * Nv];
            r3[3 * t + k] = V[F[t + 2 * (int64_t)Nt] - 1 + (int64_t)k * Nv];
            cent[3 * t + k] = (r1[3 * t + k] + r2[3 * t + k] + r3[3 * t + k]) / 3.0;  // precompute_tri_geom.m:15
        }
        area2[t] = area2_of(&r1[3 * t], &r2[3 * t], &r3[3 * t]);                 // precompute_tri_geom.m:16
        htri[t] = std::sqrt(2.0 * area2[t] / std::sqrt(3.0));                     // efie_precompute.m:19
        out->aeqTri[t] = std::sqrt((0.5 * area2[t]) / M_PI);                     // :41-42
    }
    // :24-29 nearMat (column-major, (t1,t2) at t1 + Nt*t2)
    for (int32_t t2 = 0; t2 < Nt; t2++)
        for (int32_t t1 = 0; t1 < Nt; t1++) {
            double dx = cent[3 * t1] - cent[3 * t2], dy = cent[3 * t1 + 1] - cent[3 * t2 + 1],
                   dz = cent[3 * t1 + 2] - cent[3 * t2 + 2];
            double D = std::sqrt(dx * dx + dy * dy + dz * dz);
            double th = o->near_sing_eps * 0.5 * (htri[t1] + htri[t2]);
            out->nearMat[(size_t)t1 + (size_t)Nt * t2] = D < th ? 1 : 0;
        }
    // :32-38 regular cache: r = A + u(B-A) + v(C-A), w = qw * 2A
    for (int32_t t = 0; t < Nt; t++)
        for (int i = 0; i < Nq; i++) {
            for (int k = 0; k < 3; k++) {
                double A = r1[3 * t + k], B = r2[3 * t + k], Cc = r3[3 * t + k];
                out->r_reg[i + Nq * k + (size_t)Nq * 3 * t] = A + qu[i] * (B - A) + qv[i] * (Cc - A);
            }
            out->w_reg[i + (size_t)Nq * t] = qw[i] * area2[t];
        }
    // :52-95 subdivision caches (subdivide_triangles.m child order)
    auto subdivide = [](const double *A, const double *B, const double *Cc, int depth, std::vector<double> &tris) {
        tris.assign(A, A + 3);
        tris.insert(tris.end(), B, B + 3);
        tris.insert(tris.end(), Cc, Cc + 3);
        for (int d = 0; d < depth; d++) {
            std::vector<double> nw;
            nw.reserve(tris.size() * 4);
            for (size_t s = 0; s < tris.size(); s += 9) {
                const double *A0 = &tris[s], *B0 = &tris[s + 3], *C0 = &tris[s + 6];
                double AB[3], BC[3], CA[3];
                for (int k = 0; k < 3; k++) {
                    AB[k] = 0.5 * (A0[k] + B0[k]);
                    BC[k] = 0.5 * (B0[k] + C0[k]);
                    CA[k] = 0.5 * (C0[k] + A0[k]);
                }
                const double *kids[4][3] = {{A0, AB, CA}, {AB, B0, BC}, {CA, BC, C0}, {AB, BC, CA}};
                for (auto &kd : kids)
                    for (auto *p : kd) nw.insert(nw.end(), p, p + 3);
            }
            tris.swap(nw);
        }
    };
    std::vector<double> sub;
    for (int32_t t = 0; t < Nt; t++) {
        for (int pass = 0; pass < 2; pass++) {
            const bool self = pass == 0;
            const int Ns = self ? NsS : NsN;
            subdivide(&r1[3 * t], &r2[3 * t], &r3[3 * t], self ? o->self_subdiv : o->near_subdiv, sub);
            double *R = self ? out->self_r : out->near_r;
            double *W = self ? out->self_w : out->near_w;
            for (int p = 0; p < Ns; p++) {
                const double *A = &sub[9 * p], *B = &sub[9 * p + 3], *Cc = &sub[9 * p + 6];
                double a2p = area2_of(A, B, Cc);                                  // :67 / :88
                for (int i = 0; i < Nq2; i++) {
                    for (int k = 0; k < 3; k++)
                        R[i + Nq2 * k + (size_t)Nq2 * 3 * p + (size_t)Nq2 * 3 * Ns * t] =
                            A[k] + qu2[i] * (B[k] - A[k]) + qv2[i] * (Cc[k] - A[k]);
                    W[i + (size_t)Nq2 * p + (size_t)Nq2 * Ns * t] = qw2[i] * a2p;
                }
                if (self) out->self_a[p + (size_t)NsS * t] = o->self_alpha * std::sqrt((0.5 * a2p) / M_PI);
            }
        }
    }
    out->near_alpha = o->near_alpha;
    out->self_alpha = o->self_alpha;
    return EFIE_OK;
}
