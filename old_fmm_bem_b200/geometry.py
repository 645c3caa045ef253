"""Triangulated surfaces and quadrature points for the BEM matvecs.

The reference's BEM drivers place sources at Gauss points of surface triangles
(biobem/bem3d.cxx:9-246 `gauss_trgl`, biobem/fmm_matmult.h:53-109) or at
triangle centroids (bio/main.cxx:256-282), with outward normals and weights
0.5 * hsg (twice the area times the rule weight, biobem/fmm_matmult.h:98).
No mesh files are needed here: icospheres are generated.
"""
from __future__ import annotations

import numpy as np

# 3-point rule on the reference triangle, weights summing to 1
# (biobem/bem3d.cxx:16-27): barycentric (1/6, 1/6), (2/3, 1/6), (1/6, 2/3).
GAUSS3 = np.array([[1 / 6, 1 / 6], [2 / 3, 1 / 6], [1 / 6, 2 / 3]])
GAUSS3_W = np.array([1 / 3, 1 / 3, 1 / 3])


def icosphere(subdivisions: int, radius: float = 1.0):
    """Vertices (nv, 3) and faces (nf, 3) of an icosahedron subdivided
    `subdivisions` times (20 * 4^s triangles), projected on the sphere,
    outward orientation."""
    t = (1.0 + 5 ** 0.5) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                  [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    for _ in range(subdivisions):
        nv = len(v)
        e = np.sort(np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]]), axis=1)
        uniq, inv = np.unique(e, axis=0, return_inverse=True)
        mid = v[uniq[:, 0]] + v[uniq[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        v = np.concatenate([v, mid])
        nf = len(f)
        a, b, c = (inv[:nf] + nv, inv[nf:2 * nf] + nv, inv[2 * nf:] + nv)
        f = np.concatenate([np.stack([f[:, 0], a, c], 1), np.stack([f[:, 1], b, a], 1),
                            np.stack([f[:, 2], c, b], 1), np.stack([a, b, c], 1)])
    v *= radius
    # orient outward
    n = np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 0]])
    flip = np.einsum("ij,ij->i", n, v[f].mean(axis=1)) < 0
    f[flip] = f[flip][:, [0, 2, 1]]
    return v, f


def quadrature_points(v, f, rule: str = "gauss3"):
    """Quadrature points of flat triangles: positions (3, n), outward unit
    normals (3, n), weights (n,) = area * rule weight, and the panel index of
    each point.  rule "gauss3" (3 points per panel) or "centroid" (1)."""
    p0, p1, p2 = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    cr = np.cross(p1 - p0, p2 - p0)
    area = 0.5 * np.linalg.norm(cr, axis=1)
    nrm = cr / np.linalg.norm(cr, axis=1, keepdims=True)
    if rule == "centroid":
        bary, w = np.array([[1 / 3, 1 / 3]]), np.array([1.0])
    else:
        bary, w = GAUSS3, GAUSS3_W
    pts, nms, wts, panel = [], [], [], []
    for (xi, eta), wq in zip(bary, w):
        pts.append(p0 + xi * (p1 - p0) + eta * (p2 - p0))
        nms.append(nrm)
        wts.append(area * wq)
        panel.append(np.arange(len(f)))
    # interleave so the points of one panel are consecutive
    pts = np.stack(pts, 1).reshape(-1, 3)
    nms = np.stack(nms, 1).reshape(-1, 3)
    wts = np.stack(wts, 1).reshape(-1)
    panel = np.stack(panel, 1).reshape(-1)
    return (pts.T.astype(np.float32).copy(), nms.T.astype(np.float32).copy(), wts, panel)


def bem_double_layer_problem(subdivisions: int = 6, seed: int = 0, rule: str = "gauss3"):
    """The Laplace double-layer (Gnj) matvec workload on an icosphere of radius
    1: sources = targets = quadrature points, charge = density(panel) *
    weight with densities U[-1, 1] per panel."""
    v, f = icosphere(subdivisions)
    x, n, w, panel = quadrature_points(v, f, rule)
    rng = np.random.default_rng(seed)
    dens = rng.uniform(-1.0, 1.0, len(f))
    q = (dens[panel] * w).astype(np.float32)
    return x, n, q


def geodesic_sphere(freq: int, radius: float = 1.0):
    """Class-I geodesic sphere of frequency `freq`: every icosahedron face split
    into freq^2 triangles (20 * freq^2 in all, any size, unlike the 4^s steps
    of `icosphere`), vertices projected on the sphere, outward orientation.
    Edge vertices are not merged between faces: the BEM inputs need only the
    triangles."""
    v0, f0 = icosphere(0)
    nu = int(freq)
    assert nu >= 1
    ij = np.array([(i, j) for i in range(nu + 1) for j in range(nu + 1 - i)])
    loc = {(i, j): k for k, (i, j) in enumerate(ij)}
    tri = []
    for i in range(nu):
        for j in range(nu - i):
            tri.append((loc[i, j], loc[i + 1, j], loc[i, j + 1]))
            if i + j <= nu - 2:
                tri.append((loc[i + 1, j], loc[i + 1, j + 1], loc[i, j + 1]))
    tri = np.array(tri, dtype=np.int64)
    a, b, c = v0[f0[:, 0]], v0[f0[:, 1]], v0[f0[:, 2]]
    u = ij[:, 0:1] / nu
    w = ij[:, 1:2] / nu
    pts = a[:, None, :] + u[None] * (b - a)[:, None, :] + w[None] * (c - a)[:, None, :]
    pts /= np.linalg.norm(pts, axis=2, keepdims=True)
    v = pts.reshape(-1, 3) * radius
    f = (tri[None, :, :] + (np.arange(20) * len(ij))[:, None, None]).reshape(-1, 3)
    n = np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 0]])
    flip = np.einsum("ij,ij->i", n, v[f].mean(axis=1)) < 0
    f[flip] = f[flip][:, [0, 2, 1]]
    return v, f


# Dielectric constants of the reference's BEM solve (bio/parameters.h: e1 = 4,
# e2 = 20) and the shell operator built from them (bio/main.cxx:43-48, 65)
E1, E2 = 4.0, 20.0
BEM_DIAG = (E1 + E2) / (2 * E1 * (E1 - E2))


def bem_batch_problems(nprob: int = 64, tmin: int = 2000, tmax: int = 200000, seed: int = 0):
    """Independent unit-sphere BEM problems with triangle counts log-uniform in
    [tmin, tmax] (geodesic frequency round(sqrt(T / 20))), one point per
    triangle at its centroid with outward unit normal and the panel area, as
    the reference's BEM driver places them (bio/main.cxx:256-282).  Returns a
    list of (x (3, n) float32, normals (3, n) float32, area (n,) float64)."""
    rng = np.random.default_rng(seed)
    t = np.exp(rng.uniform(np.log(tmin), np.log(tmax), nprob))
    out = []
    for T in t:
        nu = max(1, int(round((T / 20.0) ** 0.5)))
        v, f = geodesic_sphere(nu)
        x, n, w, _ = quadrature_points(v, f, "centroid")
        out.append((x, n, w))
    return out
