"""Curved 6-node boundary elements: the surface geometry of the reference's
biobem solver.

The reference's biobem driver (biobem/main.cxx:97-99) builds its surface in
three steps, restated here with the same arithmetic (single-precision storage
where the reference stores floats, double-precision evaluation where it
evaluates in double), so that every array comes out as the reference's:

* ``six_node_mesh``  -- biobem/geometry.cxx:35-162: keep the triangles of area
  above 1e-5, add the edge midpoints as nodes 4-6 of each element, merge
  coincident nodes (global numbering in order of first appearance) and list
  the elements around each node;
* ``triangle_rule``  -- biobem/bem3d.cxx:9-246 (gauss_trgl): the symmetric
  triangle quadratures of 1, 3, 4, 6, 7, 9, 12 and 13 points;
* ``element_geometry`` -- biobem/bem3d.cxx:248-542 (interp_p, elm_geom): the
  quadratic shape functions of a curved triangle whose mid-side nodes sit at
  the fractions al, be, ga of its edges, the surface metric times the rule
  weight at every quadrature point (hsg), the element areas, and the unit
  normals at the nodes (the average of the elements' normals there) with two
  tangent vectors.

``Biobem`` then runs the reference's solvation model on those elements on the
GPU: the double-layer operator of biobem/fmm_matmult.h:9-196 (node values
interpolated to the quadrature points of every element around the node, the
Laplace Gnj kernel) evaluated by the FMM plan of this package, left
preconditioned GMRES as PETSc's KSP with the shell preconditioner of
biobem/fmm_matmult.h:198-214, and the reaction energy of biobem/main.cxx:156-201.
"""
from __future__ import annotations

import numpy as np

F32 = np.float32

# The symmetric rules of biobem/bem3d.cxx:9-246 (barycentric xi, eta and
# weights summing to 1 on the reference triangle).  The tables are the
# reference's, value for value, because its outputs are what the geometry is
# pinned to -- including the 7-point rule's first abscissa, which the
# reference has as 0.797426958353087 (the published Radon value is
# 0.797426985353087).  Like the reference, the abscissas and weights are held
# in single precision.
_RULES = {
    1: ([1 / 3], [1 / 3], [1.0]),
    3: ([1 / 6, 2 / 3, 1 / 6], [1 / 6, 1 / 6, 2 / 3], [1 / 3] * 3),
    4: ([1 / 3, 1 / 5, 3 / 5, 1 / 5], [1 / 3, 1 / 5, 1 / 5, 3 / 5], [-27 / 48, 25 / 48, 25 / 48, 25 / 48]),
}


def _orbit6(al, be, ga, de, o1, o2):
    """Two three-point orbits (de, de, al) and (be, be, ga)."""
    return [de, al, de, be, ga, be], [de, de, al, be, be, ga], [o1, o1, o1, o2, o2, o2]


def _orbit12(al, be, ga, de, rh, qa, ru, o1, o2, o3):
    """Two three-point orbits and one six-point orbit (qa, ru, rh)."""
    xi = [de, al, de, be, ga, be, qa, ru, rh, qa, ru, rh]
    eta = [de, de, al, be, be, ga, ru, qa, qa, rh, rh, ru]
    return xi, eta, [o1] * 3 + [o2] * 3 + [o3] * 6


def triangle_rule(ngl: int):
    """(xi, eta, w) of the ngl-point rule as float32 arrays (gauss_trgl)."""
    if ngl in _RULES:
        xi, eta, w = _RULES[ngl]
    elif ngl == 6:
        xi, eta, w = _orbit6(0.816847572980459, 0.445948490915965, 0.108103018168070, 0.091576213509771,
                             0.109951743655322, 0.223381589678011)
    elif ngl == 7:
        xi, eta, w = _orbit6(0.797426958353087, 0.470142064105115, 0.059715871789770, 0.101286507323456,
                             0.125939180544827, 0.132394152788506)
        xi, eta, w = xi + [1 / 3], eta + [1 / 3], w + [0.225]
    elif ngl == 9:
        al, qa, rh, de, ru = 0.124949503233232, 0.165409927389841, 0.797112651860071, 0.437525248383384, 0.037477420750088
        o1, o2 = 0.205950504760887, 0.063691414286223
        xi = [de, al, de, qa, ru, rh, qa, ru, rh]
        eta = [de, de, al, ru, qa, qa, rh, rh, ru]
        w = [o1] * 3 + [o2] * 6
    elif ngl == 12:
        xi, eta, w = _orbit12(0.873821971016996, 0.249286745170910, 0.501426509658179, 0.063089014491502,
                              0.636502499121399, 0.310352451033785, 0.053145049844816,
                              0.050844906370207, 0.116786275726379, 0.082851075618374)
    elif ngl == 13:
        xi, eta, w = _orbit12(0.479308067841923, 0.065130102902216, 0.869739794195568, 0.260345966079038,
                              0.638444188569809, 0.312865496004875, 0.048690315425316,
                              0.175615257433204, 0.053347235608839, 0.077113760890257)
        xi, eta, w = xi + [1 / 3], eta + [1 / 3], w + [-0.149570044467670]
    else:
        raise ValueError("triangle rules have 1, 3, 4, 6, 7, 9, 12 or 13 points")
    return np.asarray(xi, F32), np.asarray(eta, F32), np.asarray(w, F32)


def six_node_mesh(vert, face, xyzq=None, min_area=1e-5):
    """6-node elements from a triangulation (biobem/geometry.cxx:35-162).

    vert: (nv, 3) vertex coordinates; face: (nf, 3) vertex numbers counted from
    1 (the MSMS .face convention the reference reads).  Triangles of area
    0.5 |(v2 - v0) x (v1 - v0)| <= min_area are dropped.  Returns a dict:
    ``ptr`` (nwn, 3) float32 node coordinates, ``ntr`` (nwe, 6) node numbers
    of each element (vertices 1-3, then the midpoints of edges 1-2, 2-3, 3-1),
    ``nne_ptr`` / ``nne_elm`` the elements around each node (CSR, ascending),
    and the charges ``xq`` (3, nch), ``vq`` (nch,) when xyzq is given.

    Nodes are merged when they coincide (the reference merges within 1e-6 per
    coordinate; coincident nodes of a conforming mesh are bit-identical, and
    a mesh with distinct nodes closer than that is refused here).
    """
    v = np.asarray(vert, np.float64).astype(F32)
    f = np.asarray(face, np.int64) - 1
    # edge vectors differenced in single precision, the cross product in double
    b = (v[f[:, 2]] - v[f[:, 0]]).astype(np.float64)
    d = (v[f[:, 1]] - v[f[:, 0]]).astype(np.float64)
    cx = b[:, 1] * d[:, 2] - b[:, 2] * d[:, 1]
    cy = b[:, 2] * d[:, 0] - b[:, 0] * d[:, 2]
    cz = b[:, 0] * d[:, 1] - b[:, 1] * d[:, 0]
    keep = 0.5 * np.sqrt(cx * cx + cy * cy + cz * cz) > min_area
    f = f[keep]
    xv = np.empty((len(f), 6, 3), F32)
    xv[:, :3] = v[f]
    # midpoints in single precision: 0.5 * (a + b), the sum rounded to float
    xv[:, 3] = (xv[:, 0] + xv[:, 1]) * F32(0.5)
    xv[:, 4] = (xv[:, 1] + xv[:, 2]) * F32(0.5)
    xv[:, 5] = (xv[:, 2] + xv[:, 0]) * F32(0.5)
    flat = xv.reshape(-1, 3)
    # global numbering in order of first appearance (element by element, node
    # by node), as the reference's search over the nodes found so far gives
    uniq, first, inv = np.unique(flat.view(np.dtype((np.void, 12))).ravel(), return_index=True, return_inverse=True)
    order = np.argsort(first, kind="stable")
    rank = np.empty_like(order)
    rank[order] = np.arange(len(order))
    ntr = rank[inv.ravel()].reshape(-1, 6).astype(np.int32)
    ptr = flat[first[order]]
    _check_separation(ptr)
    nwn = len(ptr)
    # elements around each node, ascending (nne of the reference)
    elm = np.repeat(np.arange(len(f), dtype=np.int32), 6)
    o = np.lexsort((elm, ntr.ravel()))
    nne_elm = elm[o]
    nne_ptr = np.zeros(nwn + 1, np.int64)
    np.add.at(nne_ptr, ntr.ravel() + 1, 1)
    nne_ptr = np.cumsum(nne_ptr)
    out = {"ptr": ptr, "ntr": ntr, "nne_ptr": nne_ptr, "nne_elm": nne_elm}
    if xyzq is not None:
        a = np.asarray(xyzq, np.float64).astype(F32)
        out["xq"] = np.ascontiguousarray(a[:, :3].T)
        out["vq"] = a[:, 3].copy()
    return out


def _check_separation(ptr, eps=1e-6):
    """Distinct nodes closer than eps in every coordinate would have been
    merged by the reference's search: refuse such meshes."""
    q = np.floor(ptr.astype(np.float64) / (2 * eps)).astype(np.int64)
    key = q[:, 0] * 73856093 ^ q[:, 1] * 19349663 ^ q[:, 2] * 83492791
    _, cnt = np.unique(key, return_counts=True)
    if np.any(cnt > 1):
        d = np.abs(ptr[:, None, :].astype(np.float64) - ptr[None, :, :]) if len(ptr) <= 4096 else None
        if d is None or np.any(np.all(d <= eps, axis=2) & ~np.eye(len(ptr), dtype=bool)):
            raise ValueError("mesh has distinct nodes within 1e-6 of each other")


def interp_p(x, y, z, al, be, ga, xi, eta):
    """Shape functions, tangents and unit normal of curved 6-node triangles at
    (xi, eta) (biobem/bem3d.cxx:248-323), vectorised over elements.

    x, y, z: (..., 6) node coordinates (double); al, be, ga: (...,) mid-node
    fractions; xi, eta broadcastable.  Returns (phi (..., 6), normal (..., 3),
    hsd (...,), dxdxi (..., 3), dxdeta (..., 3))."""
    alc, bec, gac = 1.0 - al, 1.0 - be, 1.0 - ga
    alalc, bebec, gagac = al * alc, be * bec, ga * gac
    ph2 = xi * (xi - al + eta * (al - ga) / gac) / alc
    ph3 = eta * (eta - be + xi * (be + ga - 1.0) / ga) / bec
    ph4 = xi * (1.0 - xi - eta) / alalc
    ph5 = xi * eta / gagac
    ph6 = eta * (1.0 - xi - eta) / bebec
    ph1 = 1.0 - ph2 - ph3 - ph4 - ph5 - ph6
    dph2 = (2.0 * xi - al + eta * (al - ga) / gac) / alc
    dph3 = eta * (be + ga - 1.0) / (ga * bec)
    dph4 = (1.0 - 2.0 * xi - eta) / alalc
    dph5 = eta / gagac
    dph6 = -eta / bebec
    dph1 = -dph2 - dph3 - dph4 - dph5 - dph6
    pph2 = xi * (al - ga) / (alc * gac)
    pph3 = (2.0 * eta - be + xi * (be + ga - 1.0) / ga) / bec
    pph4 = -xi / alalc
    pph5 = xi / gagac
    pph6 = (1.0 - xi - 2.0 * eta) / bebec
    pph1 = -pph2 - pph3 - pph4 - pph5 - pph6

    def comb(c, d):  # the reference's left-to-right sum c0 d0 + ... + c5 d5
        s = c[..., 0] * d[0]
        for k in range(1, 6):
            s = s + c[..., k] * d[k]
        return s

    dph = (dph1, dph2, dph3, dph4, dph5, dph6)
    pph = (pph1, pph2, pph3, pph4, pph5, pph6)
    dxi = np.stack([comb(x, dph), comb(y, dph), comb(z, dph)], -1)
    det = np.stack([comb(x, pph), comb(y, pph), comb(z, pph)], -1)
    vnx = dxi[..., 1] * det[..., 2] - det[..., 1] * dxi[..., 2]
    vny = dxi[..., 2] * det[..., 0] - det[..., 2] * dxi[..., 0]
    vnz = dxi[..., 0] * det[..., 1] - det[..., 0] * dxi[..., 1]
    hsd = np.sqrt(vnx * vnx + vny * vny + vnz * vnz)
    nrm = np.stack([vnx / hsd, vny / hsd, vnz / hsd], -1)
    phi = np.stack(np.broadcast_arrays(ph1, ph2, ph3, ph4, ph5, ph6), -1)
    return phi, nrm, hsd, dxi, det


def element_geometry(mesh, ngl=3):
    """Quadrature tables and node normals of the 6-node elements (elm_geom,
    biobem/bem3d.cxx:325-542).  Adds to (a copy of) the mesh dict:
    ``xiq``, ``etq``, ``wq`` (ngl,) float32; ``are`` (nwe,) element areas;
    ``hsg`` (nwe, ngl) surface metric x rule weight; ``phi`` (nwe, ngl, 6)
    shape functions at the quadrature points (the reference's p1..p6); ``vna``
    (nwn, 3) unit normals at the nodes; ``vta``, ``vsa`` (nwn, 3) tangents --
    all float32 like the reference's arrays."""
    g = dict(mesh)
    ptr, ntr = mesh["ptr"], mesh["ntr"]
    nwe, nwn = len(ntr), len(ptr)
    X = ptr.astype(np.float64)[ntr]  # (nwe, 6, 3)
    x, y, z = X[..., 0], X[..., 1], X[..., 2]

    def dist(a, b):
        d = X[:, a] - X[:, b]
        return np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2])

    al = 1.0 / (1.0 + dist(3, 1) / dist(3, 0))
    be = 1.0 / (1.0 + dist(5, 2) / dist(5, 0))
    ga = 1.0 / (1.0 + dist(4, 1) / dist(4, 2))
    xiq, etq, wq = triangle_rule(ngl)
    hsg = np.empty((nwe, ngl), F32)
    phi = np.empty((nwe, ngl, 6), F32)
    are = np.zeros(nwe, F32)  # summed in single precision, one rounding per point
    for j in range(ngl):
        ph, _, hsd, _, _ = interp_p(x, y, z, al, be, ga, np.float64(xiq[j]), np.float64(etq[j]))
        cf = hsd * np.float64(wq[j])
        are = (are.astype(np.float64) + cf).astype(F32)
        hsg[:, j] = cf
        phi[:, j] = ph
    are = (are.astype(np.float64) * 0.5).astype(F32)
    # normals at the element's own nodes (xi, eta) = (0,0) (1,0) (0,1) (al,0) (ga,1-ga) (0,be)
    xn = np.stack([np.zeros(nwe), np.ones(nwe), np.zeros(nwe), al, ga, np.zeros(nwe)], 1)
    en = np.stack([np.zeros(nwe), np.zeros(nwe), np.ones(nwe), np.zeros(nwe), 1.0 - ga, be], 1)
    _, nv, _, _, _ = interp_p(x[:, None, :], y[:, None, :], z[:, None, :], al[:, None], be[:, None], ga[:, None],
                              xn, en)  # (nwe, 6, 3)
    # vna[m] += normal, in element order, each addition rounded to float
    node = ntr.ravel()
    contrib = nv.reshape(-1, 3)
    o = np.argsort(node, kind="stable")  # by node, element order kept
    node_s, contrib_s = node[o], contrib[o]
    start = np.searchsorted(node_s, np.arange(nwn))
    cnt = np.bincount(node_s, minlength=nwn)
    vna = np.zeros((nwn, 3), F32)
    for k in range(int(cnt.max()) if nwn else 0):
        has = cnt > k
        idx = start[has] + k
        vna[has] = (vna[has].astype(np.float64) + contrib_s[idx]).astype(F32)
    # average, then unit length: the squares summed in single precision (the
    # reference multiplies floats), the root and the division in double
    par = cnt.astype(np.float64)[:, None]
    vna = (vna.astype(np.float64) / par).astype(F32)
    par = np.sqrt((vna[:, 0] * vna[:, 0] + vna[:, 1] * vna[:, 1] + vna[:, 2] * vna[:, 2]).astype(np.float64))
    vna = (vna.astype(np.float64) / par[:, None]).astype(F32)
    sabs = np.sqrt((vna[:, 1] * vna[:, 1] + vna[:, 2] * vna[:, 2]).astype(np.float64))
    big = sabs > 1e-3
    den = np.where(big, sabs, 1.0)
    vsa = np.zeros((nwn, 3), F32)
    vsa[:, 1] = np.where(big, vna[:, 2].astype(np.float64) / den, 1.0).astype(F32)
    vsa[:, 2] = np.where(big, -vna[:, 1].astype(np.float64) / den, 0.0).astype(F32)
    vta = np.stack([vsa[:, 1] * vna[:, 2] - vsa[:, 2] * vna[:, 1],
                    vsa[:, 2] * vna[:, 0] - vsa[:, 0] * vna[:, 2],
                    vsa[:, 0] * vna[:, 1] - vsa[:, 1] * vna[:, 0]], 1).astype(F32)
    g.update(ngl=ngl, xiq=xiq, etq=etq, wq=wq, are=are, hsg=hsg, phi=phi, vna=vna, vta=vta, vsa=vsa,
             al=al, be=be, ga=ga)
    return g


COULOMB = 332.112  # kcal/mol * Angstrom / e^2 (biobem/main.cxx:193)


def quadrature_sources(geom):
    """The quadrature points of all elements as FMM sources, element by
    element, point by point (biobem/fmm_matmult.h:112-160): positions
    sum_i phi_i x_node(i) (3, nwe * ngl) and normals sum_i phi_i vna(i)
    (interpolated, not renormalised), float32 like the reference's source
    arrays, with the node numbers (nwe * ngl, 6) and shape functions
    (nwe * ngl, 6) that interpolate node values there."""
    ptr = geom["ptr"].astype(np.float64)
    vna = geom["vna"].astype(np.float64)
    phi = geom["phi"].astype(np.float64)           # (nwe, ngl, 6)
    ntr = geom["ntr"]
    nodes = np.repeat(ntr[:, None, :], phi.shape[1], axis=1)  # (nwe, ngl, 6)

    def interp(a):  # left-to-right sum over the 6 nodes, in double
        s = a[nodes[..., 0]] * phi[..., 0:1]
        for i in range(1, 6):
            s = s + a[nodes[..., i]] * phi[..., i:i + 1]
        return s.reshape(-1, 3)

    xs = interp(ptr).astype(F32)
    ns = interp(vna).astype(F32)
    return (np.ascontiguousarray(xs.T), np.ascontiguousarray(ns.T), nodes.reshape(-1, 6),
            phi.reshape(-1, 6), geom["hsg"].astype(np.float64).reshape(-1))


class Biobem:
    """The reference's biobem solvation model (biobem/main.cxx with
    biobem/fmm_matmult.h) on 6-node curved elements, every integral an FMM
    of this package on the GPU.

    Unknown: the surface density si at the nodes.  Operator (mymatmult):

        A x = Gnj[q(x)](nodes) + s2 * x / e1 + (e1 + e2) / (e1 - e2) * x / e1,

    q(x) at quadrature point (k, j) = 0.5 * hsg_kj * sum_i phi_i x_ntr[k,i] / e1
    (the reference sums the same charges node by node, one impulse per node),
    s2 = Gnj[-0.5 * hsg](nodes) (the principal-value integral, a fixed vector).
    Preconditioner (mypcshell): y = x * 2 e1 (e1 - e2) / (e1 + e2).  Right-hand
    side: -4 pi Gni[charges](nodes, normals -vna) / e1 (biobem/main.cxx:101-123).
    Energy: 0.5 * 332.112 * sum_l q_l G[q(si)](atom l) (biobem/main.cxx:156-195).
    GMRES: restarted, left preconditioned, zero initial guess (PETSc's KSPGMRES
    defaults: restart 30, relative tolerance 1e-5), the vectors on the GPU.
    """

    def __init__(self, geom, *, e1=4.0, e2=20.0, p=12, lmax=None, precision=None):
        import torch

        import old_fmm_bem_b200 as ob
        self.ob, self.torch = ob, torch
        self.e1, self.e2 = float(e1), float(e2)
        self.geom = geom
        xs, ns, nodes, phi, hsg = quadrature_sources(geom)
        self.nwn = len(geom["ptr"])
        self.nq = xs.shape[1]
        if lmax is None:
            lmax = 2
            while lmax < 8 and self.nq / 8.0 ** lmax * 4 > 64:  # a surface fills ~1/4 of its level's boxes
                lmax += 1
        self.kw = dict(p=p, lmax=lmax, precision=ob.FP64 if precision is None else precision,
                       semantics=ob.SEM_ACCURATE, exclude_self=True)
        dev = "cuda"
        self.xn = np.ascontiguousarray(geom["ptr"].T)        # (3, nwn) nodes
        self.vna = np.ascontiguousarray(geom["vna"].T)
        self.xs, self.ns = xs, ns
        self.nodes = torch.from_numpy(nodes.astype(np.int64)).to(dev)
        self.phi = torch.from_numpy(phi).to(dev)
        self.half_hsg = torch.from_numpy(0.5 * hsg).to(dev)
        self.plan = ob.Plan(kernel=ob.LAPLACE_GNJ, **self.kw)
        self.plan.set_geometry(torch.from_numpy(self.xn).to(dev), torch.from_numpy(xs).to(dev),
                               None, torch.from_numpy(ns).to(dev))
        # principal-value term: the same sources with charges -0.5 hsg
        self.s2 = self._gnj(-self.half_hsg)
        self.iterations = 0

    def close(self):
        self.plan.close()

    def _gnj(self, q):
        out = self.torch.zeros(self.nwn, dtype=self.torch.float64, device="cuda")
        self.plan.evaluate(q.to(self.torch.float32).contiguous(), out, f64=True)
        return out

    def charges(self, x):
        """Quadrature-point charges 0.5 hsg sum_i phi_i x_node(i) / e1."""
        return self.half_hsg * (self.phi * x[self.nodes]).sum(1) / self.e1

    def matvec(self, x):
        """A x for a node vector x (torch, float64, on the GPU)."""
        e1, e2 = self.e1, self.e2
        return self._gnj(self.charges(x)) + self.s2 * x / e1 + (e1 + e2) / (e1 - e2) * x / e1

    def precond(self, x):
        return x / (self.e1 + self.e2) * (2 * self.e1 * (self.e1 - self.e2))

    def rhs(self, xq, vq):
        """-4 pi Gni(charges -> nodes, target normals -vna) / e1."""
        ob = self.ob
        with ob.Plan(kernel=ob.LAPLACE_GNI, **self.kw) as pl:
            pl.set_geometry(self.xn, xq, -self.vna, None)
            vi, _ = pl.evaluate(vq, f64=True)
        return -4 * np.pi * vi / self.e1

    def solve(self, b, *, rtol=1e-5, restart=30, max_iter=1000):
        """Left-preconditioned restarted GMRES (modified Gram-Schmidt), zero
        initial guess; returns the node densities (numpy)."""
        torch = self.torch
        b = torch.as_tensor(np.asarray(b, np.float64), device="cuda")
        x = torch.zeros_like(b)
        r = self.precond(b - self.matvec(x))
        beta0 = float(torch.linalg.norm(r))
        it = 0
        while beta0 > 0:
            beta = float(torch.linalg.norm(r))
            if beta <= rtol * beta0 or it >= max_iter:
                break
            V = [r / beta]
            H = np.zeros((restart + 1, restart))
            g = np.zeros(restart + 1)
            g[0] = beta
            k = 0
            while k < restart and it < max_iter:
                w = self.precond(self.matvec(V[k]))
                for i in range(k + 1):
                    H[i, k] = float(torch.dot(V[i], w))
                    w = w - H[i, k] * V[i]
                H[k + 1, k] = float(torch.linalg.norm(w))
                k += 1
                it += 1
                y, *_ = np.linalg.lstsq(H[:k + 1, :k], g[:k + 1], rcond=None)
                res = np.linalg.norm(g[:k + 1] - H[:k + 1, :k] @ y)
                if H[k, k - 1] == 0.0 or res <= rtol * beta0:
                    break
                V.append(w / H[k, k - 1])
            y, *_ = np.linalg.lstsq(H[:k + 1, :k], g[:k + 1], rcond=None)
            x = x + sum(float(y[i]) * V[i] for i in range(k))
            r = self.precond(b - self.matvec(x))
        self.iterations = it
        return x.cpu().numpy()

    def energy(self, si, xq, vq):
        """0.5 * 332.112 * sum_l q_l phi_l, phi the G field of the
        quadrature charges 0.5 hsg sum_i phi_i si_i / e1 at the atoms."""
        ob, torch = self.ob, self.torch
        c = self.charges(torch.as_tensor(np.asarray(si, np.float64), device="cuda")).to(torch.float32).cpu().numpy()
        with ob.Plan(kernel=ob.LAPLACE_G, **self.kw) as pl:
            pl.set_geometry(np.ascontiguousarray(xq, dtype=np.float32), self.xs)
            phi, _ = pl.evaluate(c, f64=True)
        return float(0.5 * COULOMB * np.dot(np.asarray(vq, np.float64), phi))


def solvation_energy(vert, face, xyzq, *, ngl=3, e1=4.0, e2=20.0, p=12, lmax=None, precision=None, rtol=1e-5):
    """The reference's biobem pipeline end to end: 6-node mesh, element
    geometry, right-hand side, GMRES solve, reaction energy (kcal/mol).
    face: MSMS vertex numbers counted from 1.  Returns (energy, details)."""
    geom = element_geometry(six_node_mesh(vert, face, xyzq), ngl)
    bb = Biobem(geom, e1=e1, e2=e2, p=p, lmax=lmax, precision=precision)
    try:
        b = bb.rhs(geom["xq"], geom["vq"])
        si = bb.solve(b, rtol=rtol)
        e = bb.energy(si, geom["xq"], geom["vq"])
    finally:
        bb.close()
    return e, {"nodes": bb.nwn, "elements": len(geom["ntr"]), "quadrature_points": bb.nq,
               "iterations": bb.iterations, "density": si}
