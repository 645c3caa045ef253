"""Boundary-element solvation energy on the GPU: the reference's BEM driver
(bio/main.cxx) over libfmmb's plans and batched GMRES.

The reference reads a molecular surface (MSMS .vert / .face) and the atomic
charges (.xyzq), places one collocation point per triangle at its centroid,
and solves for the surface density x of the polarisation problem

    diag * x + Gni(area/e1 .* x) = -4 pi Gni(atoms -> centroids) / e1

(bio/main.cxx:27-53 matrix, :55-70 preconditioner, :300-304 right-hand side,
:377-413 PETSc GMRES), then evaluates the reaction potential at the atoms with
the G kernel and the energy 0.5 * 332.112 * sum_l q_l phi_l (:414-498).  Here
every step runs on the GPU through the C ABI: two FMM plans (charges ->
centroids, centroids -> atoms), one Gni plan on the centroids and fmmb_gmres.

MSMS readers follow biobem/geometry.cxx:10-85 and bio/main.cxx:146-201: every
line of .vert holds x y z (first three columns), every line of .face three
1-based vertex indices, every line of .xyzq x y z q; triangles of area
<= 1e-5 are dropped.
"""
from __future__ import annotations

import numpy as np

from . import geometry

COULOMB = 332.112  # kcal/mol * Angstrom / e^2 (bio/main.cxx:498)


def read_vert(path):
    """(nv, 3) float64 vertex positions of an MSMS .vert file."""
    return np.loadtxt(path, usecols=(0, 1, 2), ndmin=2).astype(np.float64)


def read_face(path):
    """(nf, 3) int64 0-based vertex indices of an MSMS .face file."""
    return np.loadtxt(path, usecols=(0, 1, 2), dtype=np.int64, ndmin=2) - 1


def read_xyzq(path):
    """Atomic positions (3, n) float32 and charges (n,) float32 of an .xyzq file."""
    a = np.loadtxt(path, ndmin=2)
    return np.ascontiguousarray(a[:, :3].T.astype(np.float32)), a[:, 3].astype(np.float32)


def write_msms(stem, v, f, x_atoms=None, q_atoms=None):
    """Writes stem.vert / stem.face (and stem.xyzq) in the layout read above."""
    with open(stem + ".vert", "w") as fh:
        for p in v:
            fh.write(f"{p[0]:10.5f} {p[1]:10.5f} {p[2]:10.5f} 0 0 0 0 0 0\n")
    with open(stem + ".face", "w") as fh:
        for t in f:
            fh.write(f"{t[0] + 1:6d} {t[1] + 1:6d} {t[2] + 1:6d}  1      1\n")
    if x_atoms is not None:
        with open(stem + ".xyzq", "w") as fh:
            for k in range(x_atoms.shape[1]):
                fh.write(f"{x_atoms[0, k]:.6f} {x_atoms[1, k]:.6f} {x_atoms[2, k]:.6f} {q_atoms[k]:.6f}\n")


def panels(v, f):
    """Centroids (3, n) float32, unit normals (3, n) float32 and areas (n,) of
    the triangles of area > 1e-5, with the reference's orientation: the normal
    is (p2 - p0) x (p1 - p0) normalised (bio/main.cxx:256-282)."""
    p0, p1, p2 = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    c = np.cross(p2 - p0, p1 - p0)
    area = 0.5 * np.linalg.norm(c, axis=1)
    keep = area > 1e-5
    c, area = c[keep], area[keep]
    cen = (p0[keep] + p1[keep] + p2[keep]) / 3.0
    n = c / (2.0 * area)[:, None]
    return (np.ascontiguousarray(cen.T.astype(np.float32)), np.ascontiguousarray(n.T.astype(np.float32)), area)


def solvation_energy(v, f, x_atoms, q_atoms, *, e1=geometry.E1, e2=geometry.E2, p=10, precision=None,
                     lmax=None, rtol=1e-5, restart=30, max_iter=200):
    """Solvation energy (kcal/mol) of the charges in the cavity bounded by the
    triangulated surface (v, f).  Returns (energy, details dict)."""
    import old_fmm_bem_b200 as ob
    precision = ob.MIXED if precision is None else precision
    cen, nrm, area = panels(v, f)
    n = cen.shape[1]
    lo = np.minimum(cen.min(axis=1), x_atoms.min(axis=1)).astype(np.float64)
    hi = np.maximum(cen.max(axis=1), x_atoms.max(axis=1)).astype(np.float64)
    rd = float((hi - lo).max() * (1 + 1e-5))
    bbox = (float(lo[0]), float(lo[1]), float(lo[2]), rd)
    if lmax is None:
        lmax = 2
        while lmax < 8 and n / 8.0 ** lmax * 4 > 64:  # a surface fills ~1/4 of the boxes of its level
            lmax += 1
    kw = dict(p=p, lmax=lmax, precision=precision, semantics=ob.SEM_ACCURATE, exclude_self=True)
    diag = (e1 + e2) / (2 * e1 * (e1 - e2))
    # right-hand side: normal field of the charges at the centroids
    with ob.Plan(kernel=ob.LAPLACE_GNI, **kw) as pl:
        pl.set_geometry(cen, x_atoms, nrm, None, bbox=bbox)
        vi, _ = pl.evaluate(q_atoms, f64=True)
    b = -4 * np.pi * vi / e1
    # surface density
    with ob.Plan(kernel=ob.LAPLACE_GNI, **kw) as pl:
        pl.set_geometry(cen, cen, nrm, None, bbox=bbox)
        x, iters, resid = pl.gmres(b, weight=(area / e1).astype(np.float32), diag=diag, precond=1 / diag,
                                   restart=restart, max_iter=max_iter, rtol=rtol)
    # reaction potential at the atoms
    with ob.Plan(kernel=ob.LAPLACE_G, **kw) as pl:
        pl.set_geometry(x_atoms, cen, bbox=bbox)
        phi, _ = pl.evaluate((x * area / e1).astype(np.float32), f64=True)
    energy = float(0.5 * COULOMB * np.dot(q_atoms.astype(np.float64), phi))
    return energy, {"panels": n, "lmax": lmax, "iterations": iters, "rel_resid": float(resid.max()),
                    "density": x, "phi": phi}
