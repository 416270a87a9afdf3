"""CPU oracle (numpy, FP64) for the EFIE method-of-moments hot path.

TEST INFRASTRUCTURE ONLY.  This module is the checker: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import
it.  The product path (the CUDA library behind the C ABI) never calls it.

It restates, function by function, the MATLAB code of the reference
(mahmut26/Matlab-cuda-efief-vs-cpu); every function cites the file:line it
follows.  All index outputs are 1-based int32 exactly as MATLAB produces them,
all arrays are laid out as MATLAB would pass them to the MEX layer
(column-major, i.e. numpy ``order='F'``).

Parity pins: this restatement is checked against (a) the independent C
restatement in ``oracle/efie_oracle.c`` and (b) golden vectors produced by the
reference's own CUDA sources compiled unmodified against the fake-mex shim
(``oracle/Makefile`` -> ``oracle/_ref``), stored under ``tests/golden``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

MU0 = 4.0 * math.pi * 1e-7          # main_patch_gpu_mex_sweep_l.m:4
C0 = 299792458.0                      # main_patch_gpu_mex_sweep_l.m:5
EPS0 = 1.0 / (MU0 * C0 * C0)          # main_patch_gpu_mex_sweep_l.m:6


# ---------------------------------------------------------------------------
# L0: mesh and RWG topology
# ---------------------------------------------------------------------------
def linspace_matlab(d1: float, d2: float, n: int) -> np.ndarray:
    """MATLAB ``linspace``: ``d1 + (0:n1).*(d2-d1)./n1`` with both ends pinned.

    numpy's linspace divides first and multiplies after, which rounds
    differently; MATLAB multiplies first.
    """
    n1 = n - 1
    i = np.arange(n, dtype=np.float64)
    y = d1 + (i * (d2 - d1)) / n1
    y[0] = d1
    y[-1] = d2
    return y


def _plate(W, L, z, nx, ny, offset, vertex_order):
    # make_patch_with_ground_mesh.m:5-7 (patch) / :23-25 (ground)
    xs = linspace_matlab(-W / 2, W / 2, nx + 1)
    ys = linspace_matlab(-L / 2, L / 2, ny + 1)
    if vertex_order == "reference":
        # [x,y]=meshgrid(xs,ys); x(:) is column-major: y varies fastest.
        X, Y = np.meshgrid(xs, ys)          # shape (ny+1, nx+1)
        vx = X.flatten(order="F")
        vy = Y.flatten(order="F")
    elif vertex_order == "grid":
        # x fastest, consistent with the face indexing below
        X, Y = np.meshgrid(xs, ys)
        vx = X.flatten(order="C")
        vy = Y.flatten(order="C")
    else:
        raise ValueError(vertex_order)
    Vp = np.stack([vx, vy, np.full(vx.shape, z)], axis=1)
    # make_patch_with_ground_mesh.m:9-20 (faces, x-fastest indexing)
    F = np.zeros((2 * nx * ny, 3), dtype=np.int64)
    t = 0
    for j in range(1, ny + 1):
        for i in range(1, nx + 1):
            v1 = offset + (j - 1) * (nx + 1) + i
            v2 = v1 + 1
            v3 = v1 + (nx + 1)
            v4 = v3 + 1
            F[t] = (v1, v2, v4)
            F[t + 1] = (v1, v4, v3)
            t += 2
    return Vp, F


def make_patch_with_ground_mesh(Lp, Wp, Lg, Wg, h, Np_x, Np_y, Ng_x, Ng_y,
                                vertex_order="reference"):
    """make_patch_with_ground_mesh.m:1-46.

    ``vertex_order='reference'`` reproduces the reference exactly: vertices are
    numbered y-fastest (``meshgrid`` then ``(:)``, :5-7) while faces index them
    x-fastest (:13-16), which scrambles vertex positions when nx != ny.
    ``'grid'`` numbers vertices x-fastest so every face is a half rectangle.
    Returns V [Nv x 3] float64 and F [Nt x 3] int32 (1-based).
    """
    Vp, Fp = _plate(Wp, Lp, +h / 2, Np_x, Np_y, 0, vertex_order)
    Vg, Fg = _plate(Wg, Lg, -h / 2, Ng_x, Ng_y, Vp.shape[0], vertex_order)
    V = np.asfortranarray(np.vstack([Vp, Vg]))
    F = np.asfortranarray(np.vstack([Fp, Fg]).astype(np.int32))
    return V, F


def _norm3(v):
    return np.sqrt(v[..., 0] * v[..., 0] + v[..., 1] * v[..., 1] + v[..., 2] * v[..., 2])


def _cross(a, b):
    return np.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1],
                     a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                     a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], axis=-1)


def build_rwg_interior(V, F):
    """build_rwg_interior.m:1-103.

    Interior edges (shared by exactly two triangles) in the lexicographic order
    of ``unique(sort(edge),'rows')`` (:25-35); plus = first incidence in
    (triangle, local edge) order, minus = second (:47-63); sign = +1 when the
    triangle traverses the edge from the lower to the higher vertex index.
    """
    F0 = np.asarray(F, dtype=np.int64)
    Nt = F0.shape[0]
    # :10-23 directed edges (t, local edge le)
    a = np.stack([F0[:, 0], F0[:, 1], F0[:, 2]], axis=1).reshape(-1)
    b = np.stack([F0[:, 1], F0[:, 2], F0[:, 0]], axis=1).reshape(-1)
    rawTri = np.repeat(np.arange(1, Nt + 1), 3)
    lo = np.minimum(a, b)
    hi = np.maximum(a, b)
    # :25 unique rows; ic maps raw -> unique
    key = lo * (int(hi.max()) + 1) + hi
    ukey, first_idx, ic, counts = np.unique(key, return_index=True,
                                            return_inverse=True, return_counts=True)
    isInt = counts == 2
    order = np.argsort(ic, kind="stable")       # raw rows grouped by unique edge, in raw order
    starts = np.concatenate([[0], np.cumsum(counts)[:-1]])
    int_ids = np.nonzero(isInt)[0]
    r1 = order[starts[int_ids]]
    r2 = order[starts[int_ids] + 1]
    ea = lo[r1]
    eb = hi[r1]
    s1 = np.where((a[r1] == ea) & (b[r1] == eb), 1, -1)
    s2 = np.where((a[r2] == ea) & (b[r2] == eb), 1, -1)
    plusTri = rawTri[r1]
    minusTri = rawTri[r2]
    Ne = int_ids.size
    Vd = np.asarray(V, dtype=np.float64)
    ra = Vd[ea - 1]
    rb = Vd[eb - 1]
    d = rb - ra
    length = _norm3(d)
    center = 0.5 * (ra + rb)

    def opp_and_area(tris):
        tv = F0[tris - 1]                                   # [Ne,3]
        mask = (tv != ea[:, None]) & (tv != eb[:, None])
        if not np.all(mask.sum(axis=1) == 1):
            raise RuntimeError("opposite vertex not found")  # :108-110
        opp = tv[mask]
        r1_ = Vd[tv[:, 0] - 1]
        r2_ = Vd[tv[:, 1] - 1]
        r3_ = Vd[tv[:, 2] - 1]
        A = 0.5 * _norm3(_cross(r2_ - r1_, r3_ - r1_))       # :111-112
        return Vd[opp - 1], A

    rp, Ap = opp_and_area(plusTri)
    rm, Am = opp_and_area(minusTri)
    zmid = 0.5 * (Vd[:, 2].max() + Vd[:, 2].min())          # :88
    zSign = np.where(center[:, 2] > zmid, 1, -1).astype(np.int32)
    return dict(
        Ne=Ne,
        edge=np.asfortranarray(np.stack([ea, eb], axis=1).astype(np.int32)),
        plusTri=plusTri.astype(np.int32), minusTri=minusTri.astype(np.int32),
        plusSign=s1.astype(np.int32), minusSign=s2.astype(np.int32),
        rp=np.asfortranarray(rp), rm=np.asfortranarray(rm), Ap=Ap, Am=Am,
        len=length, center=np.asfortranarray(center), zSign=zSign,
    )


def pick_port_edge_by_point_and_layer(rwg, p, layerSign):
    """pick_port_edge_by_point_and_layer.m:1-11 (first minimum on ties)."""
    mask = rwg["zSign"] == layerSign
    if not mask.any():
        raise ValueError("no edge on layer %d" % layerSign)
    idx = np.nonzero(mask)[0]
    cent = rwg["center"][mask]
    d = _norm3(cent - np.asarray(p, dtype=np.float64)[None, :])
    return int(idx[int(np.argmin(d))]) + 1


def gaussian_layer_weights(V, E, edge0, spread):
    """Normalised Gaussian edge weights on the layer of ``edge0`` (1-based).

    Follows the MEX host code patch_sweep_fastquad_cuda.cu:415-459 (edge
    centres from E and V; layer = centre z above the mid-plane of edge
    centres), which equals port_weights_gaussian.m:1-29 and
    assemble_ZV_EFIE_RWG_DIFF_CPU_FAST.m:194-212 on two-plate meshes.
    """
    E0 = np.asarray(E, dtype=np.int64) - 1
    Vd = np.asarray(V, dtype=np.float64)
    c = 0.5 * (Vd[E0[:, 0]] + Vd[E0[:, 1]])
    zmid = 0.5 * (c[:, 2].min() + c[:, 2].max())
    layer = np.where(c[:, 2] > zmid, 1, -1)
    e0 = edge0 - 1
    d = _norm3(c - c[e0][None, :])
    w = np.exp(-(d / spread) * (d / spread))
    w = np.where(layer == layer[e0], w, 0.0)
    s = w.sum()
    if s < 1e-30:
        raise ValueError("mex:rhs spreadRadius too small (no weights).")
    return w / s


def rhs_edge_strip_diff_gaussian(V, E, patchEdge, groundEdge, V0, spread):
    """V = +V0/2 wPatch - V0/2 wGnd (CPU_FAST.m:184-192; fastquad.cu:589-593)."""
    wP = gaussian_layer_weights(V, E, patchEdge, spread)
    wG = gaussian_layer_weights(V, E, groundEdge, spread)
    return (V0 / 2.0) * wP + (-V0 / 2.0) * wG, wP, wG


# ---------------------------------------------------------------------------
# L1: quadrature and precompute cache
# ---------------------------------------------------------------------------
DUNAVANT7 = -7


def tri_quad_rule(order):
    """tri_quad_rule.m:1-23 on the reference triangle (0,0),(1,0),(0,1).

    Weights sum to 1/2.  ``order == DUNAVANT7`` (-7) is an addition: the
    7-point degree-5 rule of Dunavant (1985), weights scaled to sum to 1/2.
    Every other order keeps the reference meaning (1 -> 1, 2 -> 3, else -> 6).
    """
    if order == 1:
        return np.array([[1 / 3, 1 / 3]]), np.array([0.5])
    if order == 2:
        qp = np.array([[1 / 6, 1 / 6], [2 / 3, 1 / 6], [1 / 6, 2 / 3]])
        return qp, (1 / 6) * np.ones(3)
    if order == DUNAVANT7:
        return dunavant7()
    a = 0.445948490915965
    b = 0.108103018168070
    w1 = 0.111690794839005
    w2 = 0.054975871827661
    qp = np.array([[a, a], [a, 1 - 2 * a], [1 - 2 * a, a],
                   [b, b], [b, 1 - 2 * b], [1 - 2 * b, b]])
    return qp, np.array([w1, w1, w1, w2, w2, w2])


def dunavant7():
    """Dunavant (1985) degree-5, 7-point rule (barycentric orbits), sum w = 1/2.

    Centroid weight 9/40; orbits a1 = (6 - sqrt(15))/21, a2 = (6 + sqrt(15))/21
    with weights (155 - sqrt(15))/1200 and (155 + sqrt(15))/1200 (area-normalised
    weights, multiplied by 1/2 here).
    """
    s15 = math.sqrt(15.0)
    a1 = (6.0 - s15) / 21.0
    a2 = (6.0 + s15) / 21.0
    w0 = 9.0 / 40.0
    w1 = (155.0 - s15) / 1200.0
    w2 = (155.0 + s15) / 1200.0
    qp = np.array([[1 / 3, 1 / 3],
                   [a1, a1], [1 - 2 * a1, a1], [a1, 1 - 2 * a1],
                   [a2, a2], [1 - 2 * a2, a2], [a2, 1 - 2 * a2]])
    qw = 0.5 * np.array([w0, w1, w1, w1, w2, w2, w2])
    return qp, qw


def subdivide_triangles(A, B, C, depth):
    """subdivide_triangles.m:1-20; children A-AB-CA, AB-B-BC, CA-BC-C, AB-BC-CA."""
    tris = [(np.asarray(A, float), np.asarray(B, float), np.asarray(C, float))]
    for _ in range(depth):
        new = []
        for (A0, B0, C0) in tris:
            AB = 0.5 * (A0 + B0)
            BC = 0.5 * (B0 + C0)
            CA = 0.5 * (C0 + A0)
            new += [(A0, AB, CA), (AB, B0, BC), (CA, BC, C0), (AB, BC, CA)]
        tris = new
    return tris


def map_ref_to_vertices(A, B, C, qp):
    """map_ref_to_vertices.m:1-4: r = A + u(B-A) + v(C-A)."""
    u = qp[:, 0:1]
    v = qp[:, 1:2]
    return A[None, :] + u * (B - A)[None, :] + v * (C - A)[None, :]


DEFAULT_OPTS_GPU = dict(quad_order=2, near_sing_eps=1.2, self_subdiv=2, self_alpha=0.20,
                        near_subdiv=1, near_alpha=0.15, near_order=2)
DEFAULT_OPTS_ACCURATE = dict(quad_order=4, near_sing_eps=2.5, self_subdiv=2, self_alpha=0.20,
                             near_subdiv=2, near_alpha=0.15, near_order=4)


def efie_precompute_pack(V, F, opts):
    """efie_precompute.m:1-97 followed by efie_precompute_pack.m:1-59.

    Returns the packed prepack dict with MATLAB (column-major) layouts:
    r_reg [Nq,3,Nt], w_reg [Nq,Nt], nearMat uint8 [Nt,Nt], self_r
    [Nq2,3,NsS,Nt], self_w [Nq2,NsS,Nt], self_a [NsS,Nt], near_r
    [Nq2,3,NsN,Nt], near_w [Nq2,NsN,Nt], aeqTri [Nt], near_alpha, self_alpha.
    """
    o = dict(opts)
    o.setdefault("near_order", 4)                  # efie_precompute.m:5
    o.setdefault("self_subdiv", 2)                 # :45-48
    o.setdefault("self_alpha", 0.20)
    o.setdefault("near_subdiv", 2)
    o.setdefault("near_alpha", 0.15)
    qp, qw = tri_quad_rule(o["quad_order"])
    qp2, qw2 = tri_quad_rule(o["near_order"])
    Vd = np.asarray(V, dtype=np.float64)
    F0 = np.asarray(F, dtype=np.int64) - 1
    Nt = F0.shape[0]
    r1 = Vd[F0[:, 0]]
    r2 = Vd[F0[:, 1]]
    r3 = Vd[F0[:, 2]]
    cent = (r1 + r2 + r3) / 3.0                       # precompute_tri_geom.m:15
    area2 = _norm3(_cross(r2 - r1, r3 - r1))          # precompute_tri_geom.m:16
    htri = np.sqrt(2.0 * area2 / math.sqrt(3.0))      # efie_precompute.m:19
    dx = cent[:, 0:1] - cent[:, 0][None, :]
    dy = cent[:, 1:2] - cent[:, 1][None, :]
    dz = cent[:, 2:3] - cent[:, 2][None, :]
    D = np.sqrt(dx * dx + dy * dy + dz * dz)          # :24-26
    Thresh = o["near_sing_eps"] * 0.5 * (htri[:, None] + htri[None, :])
    nearMat = (D < Thresh).astype(np.uint8)           # :28-29
    Nq = qp.shape[0]
    Nq2 = qp2.shape[0]
    # :32-38 regular cache, weights include the Jacobian 2A
    u = qp[:, 0]
    v = qp[:, 1]
    r_reg = (r1[None, :, :] + u[:, None, None] * (r2 - r1)[None, :, :]
             + v[:, None, None] * (r3 - r1)[None, :, :])        # [Nq,Nt,3]
    r_reg = np.transpose(r_reg, (0, 2, 1))                        # [Nq,3,Nt]
    w_reg = qw[:, None] * area2[None, :]
    aeqTri = np.sqrt((0.5 * area2) / math.pi)                    # :41-42
    NsS = 4 ** o["self_subdiv"]
    NsN = 4 ** o["near_subdiv"]
    self_r = np.zeros((Nq2, 3, NsS, Nt))
    self_w = np.zeros((Nq2, NsS, Nt))
    self_a = np.zeros((NsS, Nt))
    near_r = np.zeros((Nq2, 3, NsN, Nt))
    near_w = np.zeros((Nq2, NsN, Nt))
    for t in range(Nt):
        A, B, C = r1[t], r2[t], r3[t]
        for p, (Ap_, Bp_, Cp_) in enumerate(subdivide_triangles(A, B, C, o["self_subdiv"])):
            a2p = float(_norm3(_cross(Bp_ - Ap_, Cp_ - Ap_)))      # :67
            self_r[:, :, p, t] = map_ref_to_vertices(Ap_, Bp_, Cp_, qp2)
            self_w[:, p, t] = qw2 * a2p
            self_a[p, t] = o["self_alpha"] * math.sqrt((0.5 * a2p) / math.pi)   # :71-73
        for p, (Ap_, Bp_, Cp_) in enumerate(subdivide_triangles(A, B, C, o["near_subdiv"])):
            a2p = float(_norm3(_cross(Bp_ - Ap_, Cp_ - Ap_)))
            near_r[:, :, p, t] = map_ref_to_vertices(Ap_, Bp_, Cp_, qp2)
            near_w[:, p, t] = qw2 * a2p
    f = np.asfortranarray
    return dict(r_reg=f(r_reg), w_reg=f(w_reg), nearMat=f(nearMat),
                self_r=f(self_r), self_w=f(self_w), self_a=f(self_a),
                near_r=f(near_r), near_w=f(near_w), aeqTri=aeqTri,
                near_alpha=float(o["near_alpha"]), self_alpha=float(o["self_alpha"]))


# ---------------------------------------------------------------------------
# L2: Z assembly (vectorised restatement of CPU_FAST, FP64)
# ---------------------------------------------------------------------------
def physics(freq, mu, eps):
    """Per-frequency constants, fastquad.cu:715-743 (principal complex sqrt)."""
    omega = 2.0 * math.pi * freq
    eps = complex(eps)
    k = omega * np.sqrt(complex(mu) * eps)
    alpha = 1j * omega * mu
    beta = 1.0 / (1j * omega * eps)
    return omega, k, alpha, beta


def _rwg_side(rwg, m, t):
    """rwg_eval_on_triangle.m:1-29 coefficients: f = c (r - v), div = 2c.

    plus side: c = s+ l/(2A+), v = r+;  minus side: c = -s- l/(2A-), v = r-.
    Returns (c, v) arrays for edges m on triangles t (0 where t is neither).
    """
    c = np.zeros(m.shape)
    v = np.zeros(m.shape + (3,))
    plus = rwg["plusTri"][m] == t
    minus = (rwg["minusTri"][m] == t) & ~plus
    lm = rwg["len"][m]
    c = np.where(plus, rwg["plusSign"][m] * (lm / (2.0 * rwg["Ap"][m])), c)
    c = np.where(minus, -rwg["minusSign"][m] * (lm / (2.0 * rwg["Am"][m])), c)
    v = np.where(plus[..., None], rwg["rp"][m], v)
    v = np.where(minus[..., None], rwg["rm"][m], v)
    return c, v


def _pair_sums(ri, wi, rj, wj, k, soft2=None, clamp=True):
    """Sums over point pairs of w_i w_j G(R) against 1, r_i, r_j and r_i.r_j.

    ri [P,Q1,3], wi [P,Q1], rj [P,Q2,3], wj [P,Q2]; returns S0 [P], S1 [P,3],
    S2 [P,3], S3 [P] (complex).  soft2 [P] (or [P,Q1,Q2]) adds a softening
    R = sqrt(R^2 + a^2); otherwise R = max(R, 1e-15).
    """
    d = ri[:, :, None, :] - rj[:, None, :, :]
    R = np.sqrt(d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1] + d[..., 2] * d[..., 2])
    if soft2 is not None:
        R = np.sqrt(R * R + soft2)
    if clamp:
        R = np.maximum(R, 1e-15)
    G = np.exp(-1j * k * R) / (4.0 * math.pi * R)
    W = wi[:, :, None] * wj[:, None, :] * G
    S0 = W.sum(axis=(1, 2))
    S1 = np.einsum("pij,pic->pc", W, ri)
    S2 = np.einsum("pij,pjc->pc", W, rj)
    S3 = np.einsum("pij,pic,pjc->p", W, ri, rj)
    return S0, S1, S2, S3


def triangle_pair_moments(prepack, k, t1, t2, kind):
    """Moments of one class of triangle pairs (arrays of 0-based t1,t2).

    kind 'regular' -> CPU_FAST.m:63-89; 'near' -> :92-136; 'self' -> :139-183.
    """
    if kind == "regular":
        r = prepack["r_reg"]
        w = prepack["w_reg"]
        ri = np.transpose(r[:, :, t1], (2, 0, 1))
        rj = np.transpose(r[:, :, t2], (2, 0, 1))
        return _pair_sums(ri, w[:, t1].T, rj, w[:, t2].T, k)
    if kind == "near":
        r = prepack["near_r"]
        w = prepack["near_w"]
        Nq2, _, Ns, _ = r.shape
        ri = np.transpose(r[:, :, :, t1], (3, 2, 0, 1)).reshape(t1.size, Ns * Nq2, 3)
        rj = np.transpose(r[:, :, :, t2], (3, 2, 0, 1)).reshape(t2.size, Ns * Nq2, 3)
        wi = np.transpose(w[:, :, t1], (2, 1, 0)).reshape(t1.size, Ns * Nq2)
        wj = np.transpose(w[:, :, t2], (2, 1, 0)).reshape(t2.size, Ns * Nq2)
        aeq = np.minimum(prepack["aeqTri"][t1], prepack["aeqTri"][t2])
        a = prepack["near_alpha"] * aeq
        return _pair_sums(ri, wi, rj, wj, k, soft2=(a * a)[:, None, None], clamp=False)
    if kind == "self":
        r = prepack["self_r"]
        w = prepack["self_w"]
        aS = prepack["self_a"]
        Nq2, _, Ns, _ = r.shape
        ri = np.transpose(r[:, :, :, t1], (3, 2, 0, 1)).reshape(t1.size, Ns * Nq2, 3)
        wi = np.transpose(w[:, :, t1], (2, 1, 0)).reshape(t1.size, Ns * Nq2)
        sub = np.repeat(np.arange(Ns), Nq2)
        same = sub[:, None] == sub[None, :]
        a2 = (aS[:, t1].T)[:, sub] ** 2                        # [P, Q] softening of sub-triangle p
        d = ri[:, :, None, :] - ri[:, None, :, :]
        R = np.sqrt(d[..., 0] ** 2 + d[..., 1] ** 2 + d[..., 2] ** 2)
        R = np.where(same[None], np.sqrt(R * R + a2[:, :, None]), np.maximum(R, 1e-15))
        G = np.exp(-1j * k * R) / (4.0 * math.pi * R)
        W = wi[:, :, None] * wi[:, None, :] * G
        S0 = W.sum(axis=(1, 2))
        S1 = np.einsum("pij,pic->pc", W, ri)
        S2 = np.einsum("pij,pjc->pc", W, ri)
        S3 = np.einsum("pij,pic,pjc->p", W, ri, ri)
        return S0, S1, S2, S3
    raise ValueError(kind)


def assemble_Z_ref(rwg, prepack, k, omega, mu, eps, chunk=200000):
    """Z of assemble_ZV_EFIE_RWG_DIFF_CPU_FAST.m:1-60 (no symmetry), vectorised.

    Z(m,n) = sum over t1 in {T+(m),T-(m)}, t2 in {T+(n),T-(n)} of
    jw mu Ivec + Isca/(jw eps), with the integral regime chosen per triangle
    pair exactly as Z_entry (:48-54): self if t1==t2, near if nearMat, else
    regular.  Ivec/Isca are formed from the per-pair moments using
    f = c (r - v), div = 2c (rwg_eval_on_triangle.m:10-28).
    """
    Ne = rwg["Ne"]
    eps = complex(eps)
    alpha = 1j * omega * mu
    beta = 1.0 / (1j * omega * eps)
    Z = np.zeros((Ne, Ne), dtype=np.complex128)
    nearMat = prepack["nearMat"]
    tri = [rwg["plusTri"].astype(np.int64) - 1, rwg["minusTri"].astype(np.int64) - 1]
    mm, nn = np.meshgrid(np.arange(Ne), np.arange(Ne), indexing="ij")
    mm = mm.reshape(-1)
    nn = nn.reshape(-1)
    for im in range(2):
        for jn in range(2):
            for s in range(0, mm.size, chunk):
                m = mm[s:s + chunk]
                n = nn[s:s + chunk]
                t1 = tri[im][m]
                t2 = tri[jn][n]
                cm, vm = _rwg_side(rwg, m, t1 + 1)
                cn, vn = _rwg_side(rwg, n, t2 + 1)
                kinds = np.where(t1 == t2, 2, np.where(nearMat[t1, t2] != 0, 1, 0))
                acc = np.zeros(m.size, dtype=np.complex128)
                for code, kind in ((0, "regular"), (1, "near"), (2, "self")):
                    sel = np.nonzero(kinds == code)[0]
                    if sel.size == 0:
                        continue
                    S0, S1, S2, S3 = triangle_pair_moments(prepack, k, t1[sel], t2[sel], kind)
                    vms = vm[sel]
                    vns = vn[sel]
                    Ivec = cm[sel] * cn[sel] * (S3 - np.einsum("pc,pc->p", S1, vns)
                                                - np.einsum("pc,pc->p", S2, vms)
                                                + np.einsum("pc,pc->p", vms, vns) * S0)
                    Isca = 4.0 * cm[sel] * cn[sel] * S0
                    acc[sel] = alpha * Ivec + beta * Isca
                Z[m, n] += acc
    return Z


def port_current(x, wP, wG, length):
    """Iport = sum((wPatch - wGnd) .* I .* len) (fastquad.cu:777-785)."""
    return np.sum((wP - wG) * length * x)


def zin_s11(Iport, V0, Z0):
    """Zin = V0/Iport, S11 = (Zin-Z0)/(Zin+Z0) (fastquad.cu:787-799)."""
    Zin = V0 / Iport
    return Zin, (Zin - Z0) / (Zin + Z0)


# ---------------------------------------------------------------------------
# Workload descriptions (synthetic inputs with the documented shapes)
# ---------------------------------------------------------------------------
@dataclass
class Design:
    Lp: float
    Wp: float
    Lg: float
    Wg: float
    h: float
    Np_x: int
    Np_y: int
    Ng_x: int
    Ng_y: int
    feed: tuple = (0.0, -7e-3)
    eps: complex = EPS0
    mu: float = MU0
    V0: float = 1.0
    Z0: float = 50.0
    freqs: np.ndarray = field(default_factory=lambda: np.linspace(2e9, 3e9, 11))
    vertex_order: str = "grid"
    opts: dict = field(default_factory=lambda: dict(DEFAULT_OPTS_GPU))


def reference_sweep_design():
    """The reference's own GPU sweep (main_patch_gpu_mex_sweep_l.m:4-56)."""
    er, tand = 2.59, 1e-4
    Lp = Wp = 20.1e-3
    h = 1.59e-3
    epsr_eff = (er + 1) / 2 + (er - 1) / 2 * (1 + 12 * h / Wp) ** (-0.5)
    eps_eff = EPS0 * epsr_eff * (1 - 1j * tand)
    inset = 13.2e-3
    return Design(Lp=Lp, Wp=Wp, Lg=0.20, Wg=0.20, h=h, Np_x=8, Np_y=6, Ng_x=12, Ng_y=12,
                  feed=(-Wp / 2 + 1e-3, -Lp / 2 + inset), eps=eps_eff,
                  freqs=linspace_matlab(1.0e9, 1.4e9, 41), vertex_order="reference",
                  opts=dict(DEFAULT_OPTS_GPU))


def build_problem(d: Design):
    """Mesh + RWG + ports + prepack + RHS for a design (the MATLAB driver steps)."""
    V, F = make_patch_with_ground_mesh(d.Lp, d.Wp, d.Lg, d.Wg, d.h, d.Np_x, d.Np_y,
                                       d.Ng_x, d.Ng_y, vertex_order=d.vertex_order)
    rwg = build_rwg_interior(V, F)
    pe = pick_port_edge_by_point_and_layer(rwg, (d.feed[0], d.feed[1], +d.h / 2), +1)
    ge = pick_port_edge_by_point_and_layer(rwg, (d.feed[0], d.feed[1], -d.h / 2), -1)
    spread = 1.5 * float(np.mean(rwg["len"]))
    pre = efie_precompute_pack(V, F, d.opts)
    b, wP, wG = rhs_edge_strip_diff_gaussian(V, rwg["edge"], pe, ge, d.V0, spread)
    return dict(V=V, F=F, rwg=rwg, patchEdge=pe, groundEdge=ge, spread=spread,
                prepack=pre, b=b, wP=wP, wG=wG, design=d)


def solve_sweep(prob, freqs=None, assemble=None):
    """Reference CPU path per frequency: Z \\ V then Zin, S11 (FP64, LAPACK).

    ``assemble(rwg, prepack, k, omega, mu, eps)`` defaults to assemble_Z_ref;
    the C restatement (oracle_c.assemble_z) is a faster drop-in.
    """
    d = prob["design"]
    freqs = d.freqs if freqs is None else freqs
    assemble = assemble_Z_ref if assemble is None else assemble
    Zin = np.zeros(len(freqs), dtype=np.complex128)
    S11 = np.zeros(len(freqs), dtype=np.complex128)
    for i, f in enumerate(freqs):
        omega, k, _, _ = physics(f, d.mu, d.eps)
        Z = assemble(prob["rwg"], prob["prepack"], k, omega, d.mu, d.eps)
        x = np.linalg.solve(Z, prob["b"].astype(np.complex128))
        Ip = port_current(x, prob["wP"], prob["wG"], prob["rwg"]["len"])
        Zin[i], S11[i] = zin_s11(Ip, d.V0, d.Z0)
    return Zin, S11


# ---------------------------------------------------------------------------
# Extraction scheme (no reference counterpart): numerical checks of the
# analytic potential integrals used by the C oracle and the product.
# ---------------------------------------------------------------------------
def _graded_gauss(s0, width, order):
    """Composite Gauss-Legendre rule on [0, 1] whose panels shrink
    geometrically towards s0 down to `width`, for integrands with a
    near-singularity of that width at s0."""
    edges = {0.0, 1.0}
    s0 = min(max(s0, 0.0), 1.0)
    edges.add(s0)
    h = max(width, 1e-15)
    while h < 1.0:
        for e in (s0 - h, s0 + h):
            if 0.0 < e < 1.0:
                edges.add(e)
        h *= 3.0
    edges = sorted(edges)
    x, w = np.polynomial.legendre.leggauss(order)
    xs, ws = [], []
    for lo, hi in zip(edges[:-1], edges[1:]):
        if hi - lo <= 0.0:
            continue
        xs.append(lo + 0.5 * (x + 1.0) * (hi - lo))
        ws.append(0.5 * w * (hi - lo))
    return np.concatenate(xs), np.concatenate(ws)


def potential_integrals_numeric(a, r, order=24):
    """I0 = int_T 1/R dS', J = int_T (r' - r)/R dS' by Duffy-transformed
    Gauss-Legendre quadrature on the three sub-triangles with apex at the
    projection rho of r.  After the transform the radial variable U carries a
    near-singularity of width |d|/|q| at U = 0 (d = height of r over the plane)
    and the edge variable V one of width dist(rho, edge)/|edge| at the foot of
    the perpendicular; both are resolved by geometrically graded composite
    rules, so the reference converges for points near edges and vertices."""
    a = np.asarray(a, dtype=np.float64)
    r = np.asarray(r, dtype=np.float64)
    n = np.cross(a[1] - a[0], a[2] - a[0])
    n /= np.linalg.norm(n)
    d = np.dot(r - a[0], n)
    rho = r - d * n
    I0 = 0.0
    J = np.zeros(3)
    for i in range(3):
        b, c = a[i], a[(i + 1) % 3]
        e = c - b
        cr = np.cross(b - rho, e)
        area2 = np.dot(cr, n)          # signed: sub-triangles outside the edge subtract
        if abs(area2) < 1e-300:
            continue
        le = np.linalg.norm(e)
        s0 = np.dot(rho - b, e) / (le * le)
        hdist = abs(area2) / le
        v, wv = _graded_gauss(s0, hdist / le, order)
        qmin = max(hdist, 1e-300)
        u, wu = _graded_gauss(0.0, max(abs(d) / (qmin + np.linalg.norm(b - rho) + le), 1e-9), order)
        U, Vv = np.meshgrid(u, v, indexing="ij")
        W = np.outer(wu, wv)
        # r' - r = (rho - r) + U q(V), formed without the cancellation of r' - r
        dv = (rho - r)[None, None, :] + U[..., None] * ((b - rho)[None, None, :] + Vv[..., None] * e[None, None, :])
        R = np.sqrt((dv ** 2).sum(-1))
        jac = U * area2
        I0 += np.sum(W * jac / R)
        J += np.einsum("ij,ijc->c", W * jac / R, dv)
    return I0, J
