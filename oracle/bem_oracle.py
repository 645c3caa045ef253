"""Dense BEM operator and GMRES in numpy -- TEST INFRASTRUCTURE ONLY.

The checker of fmmb_gmres.  The reference solves its boundary-integral system
with PETSc KSP GMRES over a shell matrix (bio/main.cxx:27-70, 377-413); PETSc is
not vendored with the reference and is absent here, and no reference test pins
a solve, so GMRES parity is unpinned: this module restates the method from its
definition (x_k minimises the preconditioned residual over x_0 plus the Krylov
space of order k; Saad and Schultz, SIAM J. Sci. Stat. Comput. 7 (1986)), with
modified Gram-Schmidt Arnoldi and a least-squares solve per cycle -- not the
CGS2 + Givens form of the product -- and it is checked against
numpy.linalg.solve.  The dense operator is the direct-sum kernel of
kernel/Gni_dir.cxx:12-17 / kernel/Gnj_dir.cxx:12-17 (accurate semantics: no
softening, zero-distance pairs skipped), checked against the oracle's C direct
sum in tests/test_oracle_pin.py.

Only tests/ and bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import numpy as np

COEF = 0.25 / np.pi


def kernel_matrix(x, kernel, nt=None, ns=None, xs=None):
    """Dense FP64 matrix of the Laplace kernels between targets x (3, n) and
    sources xs (3, m) (default x): G (kernel 0), Gni (1, target normals nt),
    Gnj (2, source normals ns); zero-distance pairs give 0."""
    x = np.asarray(x, np.float64)
    xs = x if xs is None else np.asarray(xs, np.float64)
    d = x[:, :, None] - xs[:, None, :]
    r2 = np.einsum("kij,kij->ij", d, d)
    zero = r2 == 0
    r2[zero] = 1.0
    rinv = 1.0 / np.sqrt(r2)
    if kernel == 0:
        k = COEF * rinv
    elif kernel == 1:
        k = COEF * np.einsum("kij,ki->ij", d, np.asarray(nt, np.float64)) * rinv ** 3
    else:
        k = COEF * np.einsum("kij,kj->ij", d, np.asarray(ns, np.float64)) * rinv ** 3
    k[zero] = 0.0
    return k


def bem_matrix(x, normals, weight, kernel, diag):
    """A = diag * I + K diag(weight) for targets = sources = x (the shell
    matrix of bio/main.cxx:27-53 with K = Gni there)."""
    K = kernel_matrix(x, kernel, nt=normals if kernel == 1 else None, ns=normals if kernel == 2 else None)
    return diag * np.eye(len(weight)) + K * np.asarray(weight, np.float64)[None, :]


def gmres(A, b, x0=None, *, precond=1.0, restart=30, max_iter=20, rtol=0.0):
    """Left-preconditioned restarted GMRES (M^-1 = precond * I) for A x = b.
    Returns (x, iterations, ||r_k|| / ||r_0|| of the preconditioned residual)."""
    n = len(b)
    x = np.zeros(n) if x0 is None else np.array(x0, np.float64)
    it = 0
    beta0 = None
    rel = 0.0
    while True:
        r = precond * (b - A @ x)
        beta = np.linalg.norm(r)
        if beta0 is None:
            beta0 = beta
        if beta == 0.0 or beta <= rtol * beta0 or it >= max_iter:
            rel = beta / beta0 if beta0 else 0.0
            break
        V = [r / beta]
        H = np.zeros((restart + 1, restart))
        k = 0
        done = False
        while k < restart and it < max_iter:
            w = precond * (A @ V[k])
            for i in range(k + 1):
                H[i, k] = V[i] @ w
                w = w - H[i, k] * V[i]
            H[k + 1, k] = np.linalg.norm(w)
            k += 1
            it += 1
            e1 = np.zeros(k + 1)
            e1[0] = beta
            y, *_ = np.linalg.lstsq(H[:k + 1, :k], e1, rcond=None)
            res = np.linalg.norm(e1 - H[:k + 1, :k] @ y)
            if H[k, k - 1] <= 1e-14 * np.linalg.norm(H[:k + 1, k - 1]) or res <= rtol * beta0:
                done = True
                break
            V.append(w / H[k, k - 1])
        e1 = np.zeros(k + 1)
        e1[0] = beta
        y, *_ = np.linalg.lstsq(H[:k + 1, :k], e1, rcond=None)
        x = x + np.stack(V[:k], 1) @ y
        rel = np.linalg.norm(e1 - H[:k + 1, :k] @ y) / beta0
        if done or it >= max_iter:
            break
    return x, it, rel


def solvation_energy_dense(cen, nrm, area, x_atoms, q_atoms, e1=4.0, e2=20.0):
    """The reference's BEM solvation pipeline (bio/main.cxx) with dense FP64
    matrices and a direct solve: right-hand side -4 pi Gni(atoms -> centroids)
    / e1, A = diag I + Gni diag(area / e1), reaction potential
    G(centroids -> atoms) of x * area / e1, energy 0.5 * 332.112 * q . phi."""
    diag = (e1 + e2) / (2 * e1 * (e1 - e2))
    kni = kernel_matrix(cen, 1, nt=nrm, xs=x_atoms)
    b = -4 * np.pi * (kni @ np.asarray(q_atoms, np.float64)) / e1
    A = bem_matrix(cen, nrm, np.asarray(area) / e1, 1, diag)
    x = np.linalg.solve(A, b)
    kg = kernel_matrix(x_atoms, 0, xs=cen)
    phi = kg @ (x * np.asarray(area) / e1)
    return float(0.5 * 332.112 * np.dot(np.asarray(q_atoms, np.float64), phi)), x, phi


def biobem_matvec(geom, x, e1=4.0, e2=20.0):
    """The reference's 6-node double-layer operator (biobem/fmm_matmult.h:9-196,
    mymatmult) with dense FP64 direct sums, restated in its own order: stage
    1 puts, for every node m, an impulse on m and one source at each
    quadrature point of every element around m (charge 0.5 hsg phi_m x_m / e1,
    position and normal interpolated from the element's nodes, :53-109);
    stage 2 every quadrature point with charge -0.5 hsg (:112-160), the result
    times x / e1 (:171-173); then the (e1 + e2) / (e1 - e2) x / e1 term
    (:176-178).  Targets: the nodes.  geom: old_fmm_bem_b200.mesh6 arrays."""
    ptr = geom["ptr"].astype(np.float64)
    vna = geom["vna"].astype(np.float64)
    ntr, hsg, phi = geom["ntr"], geom["hsg"].astype(np.float64), geom["phi"].astype(np.float64)
    nne_ptr, nne_elm = geom["nne_ptr"], geom["nne_elm"]
    nwn, ngl = len(ptr), hsg.shape[1]
    x = np.asarray(x, np.float64)

    def point(k, j):
        xs = np.zeros(3)
        ns = np.zeros(3)
        for i in range(6):
            xs = xs + ptr[ntr[k, i]] * phi[k, j, i]
            ns = ns + vna[ntr[k, i]] * phi[k, j, i]
        return xs.astype(np.float32), ns.astype(np.float32)

    pts = {}
    pos1, nrm1, q1 = [], [], []
    for m in range(nwn):
        for k in nne_elm[nne_ptr[m]:nne_ptr[m + 1]]:
            for j in range(ngl):
                if (k, j) not in pts:
                    pts[(k, j)] = point(k, j)
                xs, ns = pts[(k, j)]
                qint = sum(phi[k, j, i] for i in range(6) if ntr[k, i] == m)
                pos1.append(xs)
                nrm1.append(ns)
                q1.append(0.5 * hsg[k, j] * qint * x[m] / e1)
    y = kernel_matrix(ptr.T, 2, ns=np.array(nrm1).T, xs=np.array(pos1).T) @ np.array(q1)
    pos2 = np.array([pts[(k, j)][0] for k in range(len(ntr)) for j in range(ngl)])
    nrm2 = np.array([pts[(k, j)][1] for k in range(len(ntr)) for j in range(ngl)])
    s2 = kernel_matrix(ptr.T, 2, ns=nrm2.T, xs=pos2.T) @ (-0.5 * hsg.reshape(-1))
    return y + s2 * x / e1 + (e1 + e2) / (e1 - e2) * x / e1


def biobem_energy_dense(geom, e1=4.0, e2=20.0):
    """The reference's biobem pipeline (biobem/main.cxx:101-195) with dense
    FP64 matrices and a direct solve: right-hand side -4 pi Gni(charges ->
    nodes, target normals -vna) / e1, the operator of biobem_matvec as a dense
    matrix, reaction potential G(quadrature charges -> atoms), energy
    0.5 * 332.112 * sum q phi.  The operator is assembled from the quadrature
    points once (interpolation matrix times the kernel matrix), the same sums
    as biobem_matvec's node-by-node order.  Returns (energy, node densities,
    the dense operator)."""
    ptr = geom["ptr"].astype(np.float64)
    vna = geom["vna"].astype(np.float64)
    nwn = len(ptr)
    xq, vq = geom["xq"].astype(np.float64), geom["vq"].astype(np.float64)
    b = -4 * np.pi * (kernel_matrix(ptr.T, 1, nt=-vna.T, xs=xq) @ vq) / e1
    ntr, hsg, phi = geom["ntr"], geom["hsg"].astype(np.float64), geom["phi"].astype(np.float64)
    ne, ngl = hsg.shape
    pos = np.zeros((ne, ngl, 3))
    nrm = np.zeros((ne, ngl, 3))
    W = np.zeros((ne * ngl, nwn))  # node values -> quadrature charges / (0.5 hsg / e1)
    rows = np.arange(ne * ngl).reshape(ne, ngl)
    for i in range(6):
        pos += ptr[ntr[:, i]][:, None, :] * phi[:, :, i:i + 1]
        nrm += vna[ntr[:, i]][:, None, :] * phi[:, :, i:i + 1]
        np.add.at(W, (rows, np.repeat(ntr[:, i:i + 1], ngl, 1)), phi[:, :, i])
    pos = pos.reshape(-1, 3).astype(np.float32).astype(np.float64)
    nrm = nrm.reshape(-1, 3).astype(np.float32).astype(np.float64)
    w = 0.5 * hsg.reshape(-1) / e1
    K = kernel_matrix(ptr.T, 2, ns=nrm.T, xs=pos.T)
    s2 = K @ (-0.5 * hsg.reshape(-1))
    A = K @ (w[:, None] * W) + np.diag(s2 / e1 + (e1 + e2) / (e1 - e2) / e1)
    si = np.linalg.solve(A, b)
    pot = kernel_matrix(xq, 0, xs=pos.T) @ (w * (W @ si))
    return float(0.5 * 332.112 * np.dot(vq, pot)), si, A
