/*
 * CPU oracle (plain C, FP64, OpenMP) for the EFIE hot path.
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker and the timed CPU baseline.
 * Only tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py
 * load it; the product library never links it.
 *
 * It is a literal restatement of the reference's per-RWG-pair algorithm:
 *   assemble_ZV_EFIE_RWG_DIFF_CPU_FAST.m:23-60  (Z_entry over 4 triangle pairs)
 *   ...:63-89   regular cached quadrature, R = max(R, 1e-15)
 *   ...:92-136  near cached subdivision, R = sqrt(R^2 + a^2),
 *               a = near_alpha * min(aeqTri(t1), aeqTri(t2))
 *   ...:139-183 self cached subdivision, softened only when p == q
 *   rwg_eval_on_triangle.m:1-29 basis evaluation
 *   gassemble_ZV_EFIE_RWG_DIFF_GPU_FAST.cu:49-106 / :221-299 centroid variant
 *   ggassemble_ZV_EFIE_RWG_DIFF_GPU_FAST.cu:492-540 Gaussian RHS
 * All arrays use the MATLAB (column-major, 1-based index values) layout.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#include <stdlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PI_D 3.141592653589793238462643383279502884

typedef struct { double re, im; } cplx;

static inline cplx cexpj_green(double kr, double ki, double R) {
    /* exp(-j k R)/(4 pi R), k = kr + j ki  (CPU_FAST.m:82) */
    double amp = exp(ki * R), ph = kr * R, inv = 1.0 / (4.0 * PI_D * R);
    cplx g = { amp * cos(ph) * inv, -amp * sin(ph) * inv };
    return g;
}

typedef struct {
    int Ne, Nt, Nq, Nq2, NsS, NsN;
    const int32_t *plusTri, *minusTri, *plusSign, *minusSign;
    const double *rp, *rm, *Ap, *Am, *len;
    const double *r_reg, *w_reg;
    const uint8_t *nearMat;
    const double *self_r, *self_w, *self_a, *near_r, *near_w, *aeqTri;
    double near_alpha;
} oracle_in;

/* rwg_eval_on_triangle.m:10-28 */
static inline void rwg_eval(const oracle_in *in, int m, int t, const double r[3], double f[3], double *dv) {
    int Ne = in->Ne;
    if (t == in->plusTri[m]) {
        double s = in->plusSign[m], l = in->len[m], A = in->Ap[m];
        double sc = s * (l / (2.0 * A));
        for (int c = 0; c < 3; c++) f[c] = sc * (r[c] - in->rp[m + c * Ne]);
        *dv = s * (l / A);
        return;
    }
    if (t == in->minusTri[m]) {
        double s = in->minusSign[m], l = in->len[m], A = in->Am[m];
        double sc = s * (l / (2.0 * A));
        for (int c = 0; c < 3; c++) f[c] = sc * (in->rm[m + c * Ne] - r[c]);
        *dv = s * (-(l / A));
        return;
    }
    f[0] = f[1] = f[2] = 0.0;
    *dv = 0.0;
}

/* one point-pair contribution */
static inline void accum(const oracle_in *in, int m, int n, int t1, int t2,
                         const double ri[3], double wi, const double rj[3], double wj,
                         double R, double kr, double ki, cplx *Iv, cplx *Is) {
    double fm[3], fn[3], dm, dn;
    rwg_eval(in, m, t1, ri, fm, &dm);
    rwg_eval(in, n, t2, rj, fn, &dn);
    cplx G = cexpj_green(kr, ki, R);
    double w = wi * wj;
    double ff = fm[0] * fn[0] + fm[1] * fn[1] + fm[2] * fn[2];
    double dd = dm * dn;
    Iv->re += G.re * (w * ff); Iv->im += G.im * (w * ff);
    Is->re += G.re * (w * dd); Is->im += G.im * (w * dd);
}

static inline double dist3(const double a[3], const double b[3]) {
    double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
    return sqrt(dx * dx + dy * dy + dz * dz);
}

/* CPU_FAST.m:63-89 (t1, t2 1-based) */
static void pair_regular(const oracle_in *in, int m, int n, int t1, int t2, double kr, double ki, cplx *Iv, cplx *Is) {
    int Nq = in->Nq, a = t1 - 1, b = t2 - 1;
    for (int i = 0; i < Nq; i++) {
        double ri[3] = { in->r_reg[i + Nq * 0 + Nq * 3 * a], in->r_reg[i + Nq * 1 + Nq * 3 * a], in->r_reg[i + Nq * 2 + Nq * 3 * a] };
        double wi = in->w_reg[i + Nq * a];
        for (int j = 0; j < Nq; j++) {
            double rj[3] = { in->r_reg[j + Nq * 0 + Nq * 3 * b], in->r_reg[j + Nq * 1 + Nq * 3 * b], in->r_reg[j + Nq * 2 + Nq * 3 * b] };
            double wj = in->w_reg[j + Nq * b];
            double R = dist3(ri, rj);
            if (R < 1e-15) R = 1e-15;
            accum(in, m, n, t1, t2, ri, wi, rj, wj, R, kr, ki, Iv, Is);
        }
    }
}

/* CPU_FAST.m:92-136 */
static void pair_near(const oracle_in *in, int m, int n, int t1, int t2, double kr, double ki, cplx *Iv, cplx *Is) {
    int Nq2 = in->Nq2, Ns = in->NsN, a = t1 - 1, b = t2 - 1;
    double aeq = in->aeqTri[a] < in->aeqTri[b] ? in->aeqTri[a] : in->aeqTri[b];
    double as = in->near_alpha * aeq;
    const double *R1 = in->near_r, *W1 = in->near_w;
    for (int p = 0; p < Ns; p++)
        for (int i = 0; i < Nq2; i++) {
            size_t bi = (size_t)i + (size_t)Nq2 * 3 * p + (size_t)Nq2 * 3 * Ns * a;
            double ri[3] = { R1[bi], R1[bi + Nq2], R1[bi + 2 * Nq2] };
            double wi = W1[i + Nq2 * p + (size_t)Nq2 * Ns * a];
            for (int q = 0; q < Ns; q++)
                for (int j = 0; j < Nq2; j++) {
                    size_t bj = (size_t)j + (size_t)Nq2 * 3 * q + (size_t)Nq2 * 3 * Ns * b;
                    double rj[3] = { R1[bj], R1[bj + Nq2], R1[bj + 2 * Nq2] };
                    double wj = W1[j + Nq2 * q + (size_t)Nq2 * Ns * b];
                    double R = dist3(ri, rj);
                    R = sqrt(R * R + as * as);
                    accum(in, m, n, t1, t2, ri, wi, rj, wj, R, kr, ki, Iv, Is);
                }
        }
}

/* CPU_FAST.m:139-183 */
static void pair_self(const oracle_in *in, int m, int n, int t, double kr, double ki, cplx *Iv, cplx *Is) {
    int Nq2 = in->Nq2, Ns = in->NsS, a = t - 1;
    const double *R1 = in->self_r, *W1 = in->self_w;
    for (int p = 0; p < Ns; p++) {
        double aS = in->self_a[p + Ns * a];
        for (int i = 0; i < Nq2; i++) {
            size_t bi = (size_t)i + (size_t)Nq2 * 3 * p + (size_t)Nq2 * 3 * Ns * a;
            double ri[3] = { R1[bi], R1[bi + Nq2], R1[bi + 2 * Nq2] };
            double wi = W1[i + Nq2 * p + (size_t)Nq2 * Ns * a];
            for (int q = 0; q < Ns; q++)
                for (int j = 0; j < Nq2; j++) {
                    size_t bj = (size_t)j + (size_t)Nq2 * 3 * q + (size_t)Nq2 * 3 * Ns * a;
                    double rj[3] = { R1[bj], R1[bj + Nq2], R1[bj + 2 * Nq2] };
                    double wj = W1[j + Nq2 * q + (size_t)Nq2 * Ns * a];
                    double R = dist3(ri, rj);
                    if (p == q) R = sqrt(R * R + aS * aS);
                    else if (R < 1e-15) R = 1e-15;
                    accum(in, m, n, t, t, ri, wi, rj, wj, R, kr, ki, Iv, Is);
                }
        }
    }
}

/*
 * Z (interleaved complex128, column-major Ne x Ne) for rows/cols in
 * [col0, col1) of the column range only (a bounded sample when col1 < Ne).
 * Returns 0.
 */
int oracle_assemble_z(int Ne, int Nt, int Nq, int Nq2, int NsS, int NsN,
                      const int32_t *plusTri, const int32_t *minusTri,
                      const int32_t *plusSign, const int32_t *minusSign,
                      const double *rp, const double *rm,
                      const double *Ap, const double *Am, const double *len,
                      const double *r_reg, const double *w_reg, const uint8_t *nearMat,
                      const double *self_r, const double *self_w, const double *self_a,
                      const double *near_r, const double *near_w, const double *aeqTri,
                      double near_alpha,
                      double k_re, double k_im, double omega, double mu,
                      double eps_re, double eps_im,
                      int col0, int col1, double *Z, int nthreads) {
    oracle_in in = { Ne, Nt, Nq, Nq2, NsS, NsN, plusTri, minusTri, plusSign, minusSign,
                     rp, rm, Ap, Am, len, r_reg, w_reg, nearMat, self_r, self_w, self_a,
                     near_r, near_w, aeqTri, near_alpha };
    /* alpha = j w mu ; beta = 1/(j w eps)  (fastquad.cu:738-743) */
    double al_re = 0.0, al_im = omega * mu;
    double dre = -omega * eps_im, dim = omega * eps_re, d2 = dre * dre + dim * dim;
    double be_re = dre / d2, be_im = -dim / d2;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
#pragma omp parallel for schedule(dynamic, 1)
    for (int n = col0; n < col1; n++) {
        int tn[2] = { plusTri[n], minusTri[n] };
        for (int m = 0; m < Ne; m++) {
            int tm[2] = { plusTri[m], minusTri[m] };
            double zr = 0.0, zi = 0.0;
            for (int im = 0; im < 2; im++) {
                int t1 = tm[im];
                if (t1 == 0) continue;
                for (int jn = 0; jn < 2; jn++) {
                    int t2 = tn[jn];
                    if (t2 == 0) continue;
                    cplx Iv = { 0, 0 }, Is = { 0, 0 };
                    if (t1 == t2) pair_self(&in, m, n, t1, k_re, k_im, &Iv, &Is);
                    else if (nearMat[(size_t)(t1 - 1) + (size_t)Nt * (t2 - 1)])
                        pair_near(&in, m, n, t1, t2, k_re, k_im, &Iv, &Is);
                    else pair_regular(&in, m, n, t1, t2, k_re, k_im, &Iv, &Is);
                    /* Zmn += alpha*Ivec + beta*Isca (CPU_FAST.m:56) */
                    zr += al_re * Iv.re - al_im * Iv.im + be_re * Is.re - be_im * Is.im;
                    zi += al_re * Iv.im + al_im * Iv.re + be_re * Is.im + be_im * Is.re;
                }
            }
            size_t o = 2 * ((size_t)m + (size_t)Ne * n);
            Z[o] = zr;
            Z[o + 1] = zi;
        }
    }
    return 0;
}

/*
 * Centroid (one point per triangle, weight = area) assembly:
 * gassemble_ZV_EFIE_RWG_DIFF_GPU_FAST.cu:221-299 (host side data) and
 * :49-106 (kernel).  Softening a = selfAlpha*sqrt(A/pi) only when the two
 * triangles are the same; R clamped to 1e-15 afterwards.
 */
int oracle_assemble_centroid(int Nv, int Nt, int Ne, const double *V, const int32_t *F,
                             const int32_t *plusTri, const int32_t *minusTri,
                             const int32_t *plusSign, const int32_t *minusSign,
                             const double *rp, const double *rm,
                             const double *Ap, const double *Am, const double *len,
                             double selfAlpha, double k_re, double k_im, double omega, double mu,
                             double eps_re, double eps_im, double *Z, int nthreads) {
    double al_im = omega * mu;
    double dre = -omega * eps_im, dim = omega * eps_re, d2 = dre * dre + dim * dim;
    double be_re = dre / d2, be_im = -dim / d2;
    double *cent = (double *)calloc((size_t)Nt * 4, sizeof(double)); /* cx,cy,cz,asoft */
    double *side = (double *)calloc((size_t)Ne * 2 * 9, sizeof(double)); /* pos3,f3,div,w,t */
    if (!cent || !side) { free(cent); free(side); return -1; }
    for (int t = 0; t < Nt; t++) {
        int i1 = F[t] - 1, i2 = F[t + Nt] - 1, i3 = F[t + 2 * Nt] - 1;
        if (i1 < 0 || i2 < 0 || i3 < 0 || i1 >= Nv || i2 >= Nv || i3 >= Nv) { free(cent); free(side); return -2; }
        double r1[3], r2[3], r3[3];
        for (int c = 0; c < 3; c++) { r1[c] = V[i1 + c * Nv]; r2[c] = V[i2 + c * Nv]; r3[c] = V[i3 + c * Nv]; }
        for (int c = 0; c < 3; c++) cent[4 * t + c] = (r1[c] + r2[c] + r3[c]) / 3.0;
        double e1[3] = { r2[0] - r1[0], r2[1] - r1[1], r2[2] - r1[2] };
        double e2[3] = { r3[0] - r1[0], r3[1] - r1[1], r3[2] - r1[2] };
        double cx = e1[1] * e2[2] - e1[2] * e2[1], cy = e1[2] * e2[0] - e1[0] * e2[2], cz = e1[0] * e2[1] - e1[1] * e2[0];
        double A = 0.5 * sqrt(cx * cx + cy * cy + cz * cz);
        cent[4 * t + 3] = selfAlpha * sqrt(A / PI_D);        /* gassemble.cu:246 */
    }
    for (int e = 0; e < Ne; e++) {
        for (int sd = 0; sd < 2; sd++) {
            double *o = side + (size_t)(2 * e + sd) * 9;
            int t = sd == 0 ? plusTri[e] : minusTri[e];
            double A = sd == 0 ? Ap[e] : Am[e];
            o[8] = t;
            o[7] = t > 0 ? A : 0.0;
            for (int c = 0; c < 3; c++) o[c] = t > 0 ? cent[4 * (t - 1) + c] : 0.0;
            if (t > 0 && A > 0) {
                double l = len[e];
                int s = sd == 0 ? plusSign[e] : minusSign[e];
                double sc = (double)s * (l / (2.0 * A));
                for (int c = 0; c < 3; c++)
                    o[3 + c] = sd == 0 ? sc * (o[c] - rp[e + c * Ne]) : sc * (rm[e + c * Ne] - o[c]);
                o[6] = sd == 0 ? (double)s * (l / A) : (double)s * (-(l / A));
            } else {
                o[3] = o[4] = o[5] = o[6] = 0.0;
            }
        }
    }
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
#pragma omp parallel for schedule(static)
    for (int n = 0; n < Ne; n++)
        for (int m = 0; m < Ne; m++) {
            double zr = 0.0, zi = 0.0;
            for (int sa = 0; sa < 2; sa++) {
                const double *a = side + (size_t)(2 * m + sa) * 9;
                if (a[7] == 0.0 || a[8] == 0.0) continue;
                for (int sb = 0; sb < 2; sb++) {
                    const double *b = side + (size_t)(2 * n + sb) * 9;
                    if (b[7] == 0.0 || b[8] == 0.0) continue;
                    double R = sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]) + (a[2] - b[2]) * (a[2] - b[2]));
                    if (a[8] == b[8]) { double s = cent[4 * ((int)a[8] - 1) + 3]; R = sqrt(R * R + s * s); }
                    if (R < 1e-15) R = 1e-15;
                    cplx G = cexpj_green(k_re, k_im, R);
                    double w = a[7] * b[7];
                    double ff = (a[3] * b[3] + a[4] * b[4] + a[5] * b[5]) * w, dd = (a[6] * b[6]) * w;
                    double vr = G.re * ff, vi = G.im * ff, sr = G.re * dd, si = G.im * dd;
                    /* alpha*term_vec + beta*term_sca, alpha = j*al_im */
                    zr += -al_im * vi + be_re * sr - be_im * si;
                    zi += al_im * vr + be_re * si + be_im * sr;
                }
            }
            size_t o = 2 * ((size_t)m + (size_t)Ne * n);
            Z[o] = zr;
            Z[o + 1] = zi;
        }
    free(cent);
    free(side);
    return 0;
}

/* ====================================================================== */
/* Extraction scheme (no reference counterpart): Dunavant 7-point rule on   */
/* every triangle; on self and vertex-adjacent pairs the kernel is split as */
/* G = 1/(4 pi R) + (exp(-jkR) - 1)/(4 pi R): the first term integrated     */
/* analytically over the inner triangle (Wilton et al. 1984; Graglia 1993), */
/* the second (smooth) term by the 7x7 rule.  For a pair the outer triangle */
/* is the lower index, the inner the higher, so Z is symmetric.             */
/* ====================================================================== */

/* I0 = int_T 1/R dS', J = int_T (r' - r)/R dS' for the triangle a[0..2]. */
void oracle_potential_integrals(const double a[3][3], const double r[3], double *I0, double J[3]) {
    double e1[3], e2[3], n[3];
    for (int c = 0; c < 3; c++) { e1[c] = a[1][c] - a[0][c]; e2[c] = a[2][c] - a[0][c]; }
    n[0] = e1[1] * e2[2] - e1[2] * e2[1];
    n[1] = e1[2] * e2[0] - e1[0] * e2[2];
    n[2] = e1[0] * e2[1] - e1[1] * e2[0];
    double nn = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    for (int c = 0; c < 3; c++) n[c] /= nn;
    double d = n[0] * (r[0] - a[0][0]) + n[1] * (r[1] - a[0][1]) + n[2] * (r[2] - a[0][2]);
    double ad = fabs(d);
    double rho[3] = { r[0] - d * n[0], r[1] - d * n[1], r[2] - d * n[2] };
    double s0 = 0.0, v[3] = { 0.0, 0.0, 0.0 };
    for (int i = 0; i < 3; i++) {
        const double *p = a[i], *q = a[(i + 1) % 3];
        double l[3] = { q[0] - p[0], q[1] - p[1], q[2] - p[2] };
        double ll = sqrt(l[0] * l[0] + l[1] * l[1] + l[2] * l[2]);
        for (int c = 0; c < 3; c++) l[c] /= ll;
        double u[3] = { l[1] * n[2] - l[2] * n[1], l[2] * n[0] - l[0] * n[2], l[0] * n[1] - l[1] * n[0] };
        double P0 = (p[0] - rho[0]) * u[0] + (p[1] - rho[1]) * u[1] + (p[2] - rho[2]) * u[2];
        double lp = (q[0] - rho[0]) * l[0] + (q[1] - rho[1]) * l[1] + (q[2] - rho[2]) * l[2];
        double lm = (p[0] - rho[0]) * l[0] + (p[1] - rho[1]) * l[1] + (p[2] - rho[2]) * l[2];
        double R02 = P0 * P0 + d * d;
        double Rp = sqrt(R02 + lp * lp), Rm = sqrt(R02 + lm * lm);
        double f;
        if (R02 < 1e-30 * (lp * lp + lm * lm)) f = 0.0;            /* r on the edge line: terms vanish */
        else {
            /* f = log((Rp + lp)/(Rm + lm)); R + l = R02/(R - l) where l < 0 avoids the cancellation */
            double np_ = lp >= 0.0 ? Rp + lp : R02 / (Rp - lp);
            double nm_ = lm >= 0.0 ? Rm + lm : R02 / (Rm - lm);
            f = log(np_ / nm_);
        }
        double beta = 0.0;
        if (ad > 0.0) beta = atan(P0 * lp / (R02 + ad * Rp)) - atan(P0 * lm / (R02 + ad * Rm));
        s0 += P0 * f - ad * beta;
        double t = R02 * f + lp * Rp - lm * Rm;
        for (int c = 0; c < 3; c++) v[c] += 0.5 * u[c] * t;
    }
    *I0 = s0;
    for (int c = 0; c < 3; c++) J[c] = v[c] - d * n[c] * s0;
}

/* (exp(-jkR) - 1)/(4 pi R) without cancellation; its limit -jk/(4 pi) at R = 0 */
static inline cplx smooth_green(double kr, double ki, double R) {
    cplx g;
    if (R == 0.0) { g.re = ki / (4.0 * PI_D); g.im = -kr / (4.0 * PI_D); return g; }
    double ph = kr * R, s = sin(ph), h = sin(0.5 * ph);
    double em = expm1(ki * R), e = 1.0 + em;
    /* e^{kiR}(cos - j sin) - 1 = em*cos + (cos - 1) - j e sin, cos - 1 = -2 sin^2(ph/2) */
    double c = cos(ph);
    g.re = (em * c - 2.0 * h * h) / (4.0 * PI_D * R);
    g.im = (-e * s) / (4.0 * PI_D * R);
    return g;
}

typedef struct {
    int Nv, Nt, Ne;
    const double *V; const int32_t *F;
    const int32_t *plusTri, *minusTri, *plusSign, *minusSign;
    const double *rp, *rm, *Ap, *Am, *len;
    double qu[7], qv[7], qw[7];
    int nq;
} ext_in;

static void tri_vertices(const ext_in *in, int t, double a[3][3]) {
    for (int j = 0; j < 3; j++) {
        int v = in->F[t + (size_t)j * in->Nt] - 1;
        for (int c = 0; c < 3; c++) a[j][c] = in->V[v + (size_t)c * in->Nv];
    }
}

/* rule points of triangle t (map_ref_to_vertices.m) and weights times 2A */
static void tri_points(const ext_in *in, int t, double pts[7][3], double w[7]) {
    double a[3][3];
    tri_vertices(in, t, a);
    double e1[3], e2[3];
    for (int c = 0; c < 3; c++) { e1[c] = a[1][c] - a[0][c]; e2[c] = a[2][c] - a[0][c]; }
    double cx = e1[1] * e2[2] - e1[2] * e2[1], cy = e1[2] * e2[0] - e1[0] * e2[2], cz = e1[0] * e2[1] - e1[1] * e2[0];
    double a2 = sqrt(cx * cx + cy * cy + cz * cz);
    for (int i = 0; i < in->nq; i++) {
        for (int c = 0; c < 3; c++) pts[i][c] = a[0][c] + in->qu[i] * e1[c] + in->qv[i] * e2[c];
        w[i] = in->qw[i] * a2;
    }
}

static int share_vertex(const ext_in *in, int t1, int t2) {
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            if (in->F[t1 + (size_t)i * in->Nt] == in->F[t2 + (size_t)j * in->Nt]) return 1;
    return 0;
}

/* RWG basis of edge m on triangle t (1-based): f = c (r - v), div = 2c */
static void basis(const ext_in *in, int m, int t, double *c, double v[3]) {
    int Ne = in->Ne;
    if (t == in->plusTri[m]) {
        *c = in->plusSign[m] * (in->len[m] / (2.0 * in->Ap[m]));
        for (int k = 0; k < 3; k++) v[k] = in->rp[m + k * Ne];
    } else {
        *c = -in->minusSign[m] * (in->len[m] / (2.0 * in->Am[m]));
        for (int k = 0; k < 3; k++) v[k] = in->rm[m + k * Ne];
    }
}

/* Ivec, Isca of edges mo (outer triangle to) and mi (inner triangle ti) */
static void pair_extract(const ext_in *in, int mo, int to, int mi, int ti, double kr, double ki,
                         cplx *Iv, cplx *Is) {
    double po[7][3], wo[7], pi_[7][3], wi[7];
    tri_points(in, to - 1, po, wo);
    tri_points(in, ti - 1, pi_, wi);
    double co, vo[3], ci, vi[3];
    basis(in, mo, to, &co, vo);
    basis(in, mi, ti, &ci, vi);
    int sing = (to == ti) || share_vertex(in, to - 1, ti - 1);
    double at[3][3];
    tri_vertices(in, ti - 1, at);
    for (int p = 0; p < in->nq; p++) {
        double fo[3] = { co * (po[p][0] - vo[0]), co * (po[p][1] - vo[1]), co * (po[p][2] - vo[2]) };
        double dvo = 2.0 * co;
        if (sing) {
            double I0, J[3];
            oracle_potential_integrals(at, po[p], &I0, J);
            /* int f_i / R = c_i (J + (r - v_i) I0), int div_i / R = 2 c_i I0 */
            double g[3] = { ci * (J[0] + (po[p][0] - vi[0]) * I0), ci * (J[1] + (po[p][1] - vi[1]) * I0),
                            ci * (J[2] + (po[p][2] - vi[2]) * I0) };
            Iv->re += wo[p] * (fo[0] * g[0] + fo[1] * g[1] + fo[2] * g[2]) / (4.0 * PI_D);
            Is->re += wo[p] * dvo * (2.0 * ci * I0) / (4.0 * PI_D);
        }
        for (int q = 0; q < in->nq; q++) {
            double fi[3] = { ci * (pi_[q][0] - vi[0]), ci * (pi_[q][1] - vi[1]), ci * (pi_[q][2] - vi[2]) };
            double R = dist3(po[p], pi_[q]);
            cplx G;
            if (sing) G = smooth_green(kr, ki, R);
            else G = cexpj_green(kr, ki, R < 1e-15 ? 1e-15 : R);
            double w = wo[p] * wi[q];
            double ff = fo[0] * fi[0] + fo[1] * fi[1] + fo[2] * fi[2], dd = dvo * 2.0 * ci;
            Iv->re += G.re * (w * ff); Iv->im += G.im * (w * ff);
            Is->re += G.re * (w * dd); Is->im += G.im * (w * dd);
        }
    }
}

int oracle_assemble_z_extract(int Nv, int Nt, int Ne, const double *V, const int32_t *F,
                              const int32_t *plusTri, const int32_t *minusTri,
                              const int32_t *plusSign, const int32_t *minusSign,
                              const double *rp, const double *rm, const double *Ap, const double *Am,
                              const double *len, int nq, const double *qu, const double *qv, const double *qw,
                              double k_re, double k_im, double omega, double mu, double eps_re, double eps_im,
                              int col0, int col1, double *Z, int nthreads) {
    ext_in in = { Nv, Nt, Ne, V, F, plusTri, minusTri, plusSign, minusSign, rp, rm, Ap, Am, len,
                  {0}, {0}, {0}, nq };
    if (nq > 7) return -1;
    for (int i = 0; i < nq; i++) { in.qu[i] = qu[i]; in.qv[i] = qv[i]; in.qw[i] = qw[i]; }
    double al_im = omega * mu;
    double dre = -omega * eps_im, dim = omega * eps_re, d2 = dre * dre + dim * dim;
    double be_re = dre / d2, be_im = -dim / d2;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
#pragma omp parallel for schedule(dynamic, 1)
    for (int n = col0; n < col1; n++) {
        int tn[2] = { plusTri[n], minusTri[n] };
        for (int m = 0; m < Ne; m++) {
            int tm[2] = { plusTri[m], minusTri[m] };
            double zr = 0.0, zi = 0.0;
            for (int a = 0; a < 2; a++) {
                if (tm[a] == 0) continue;
                for (int b = 0; b < 2; b++) {
                    if (tn[b] == 0) continue;
                    cplx Iv = { 0, 0 }, Is = { 0, 0 };
                    if (tm[a] == tn[b]) {
                        /* self pair: the outer-numeric / inner-analytic split is not symmetric in
                           the two basis functions; the mean of both orders keeps Z symmetric */
                        cplx Iv2 = { 0, 0 }, Is2 = { 0, 0 };
                        pair_extract(&in, m, tm[a], n, tn[b], k_re, k_im, &Iv, &Is);
                        pair_extract(&in, n, tn[b], m, tm[a], k_re, k_im, &Iv2, &Is2);
                        Iv.re = 0.5 * (Iv.re + Iv2.re); Iv.im = 0.5 * (Iv.im + Iv2.im);
                        Is.re = 0.5 * (Is.re + Is2.re); Is.im = 0.5 * (Is.im + Is2.im);
                    } else if (tm[a] < tn[b]) {
                        pair_extract(&in, m, tm[a], n, tn[b], k_re, k_im, &Iv, &Is);
                    } else {
                        pair_extract(&in, n, tn[b], m, tm[a], k_re, k_im, &Iv, &Is);
                    }
                    zr += -al_im * Iv.im + be_re * Is.re - be_im * Is.im;
                    zi += al_im * Iv.re + be_re * Is.im + be_im * Is.re;
                }
            }
            size_t o = 2 * ((size_t)m + (size_t)Ne * n);
            Z[o] = zr;
            Z[o + 1] = zi;
        }
    }
    return 0;
}
