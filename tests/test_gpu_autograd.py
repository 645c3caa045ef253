"""The hand-written adjoint behind torch.autograd (old_fmm_bem_b200/autograd.py)
against the FP64 direct-sum gradient and central finite differences.

L = sum_i w_i pot_i.  Direct-sum references (oracle, FP64, no softening, zero
distance pairs skipped):
  dL/dq   = G(targets = x_s, sources = x_t, charges = w)          (G symmetric)
  dL/dx_t = w * grad pot(x_t),   dL/dx_s = q * grad psi(x_s),  psi = G(x_s <- x_t, w)
and for the normal-derivative kernels dL/dq = -Gnj / -Gni with the sets swapped.
Tolerances: 2e-5 relative (FMM truncation at p = 12 is ~1e-6 on potentials,
a few 1e-6 on fields); finite differences (h = 1e-3) to 1e-2.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def ag():
    from old_fmm_bem_b200 import autograd, build
    build.build()
    return autograd


@pytest.mark.parametrize("precision", [0, 1])
def test_laplace_g_gradients_vs_direct(precision, ag, oracle):
    rng = np.random.default_rng(5)
    ni, nj = 3000, 4000
    xt = rng.random((3, ni), dtype=np.float32)
    xs = rng.random((3, nj), dtype=np.float32)
    q = rng.standard_normal(nj).astype(np.float32)
    w = rng.standard_normal(ni)
    Xt = torch.tensor(xt, device="cuda", requires_grad=True)
    Xs = torch.tensor(xs, device="cuda", requires_grad=True)
    Q = torch.tensor(q, device="cuda", dtype=torch.float64, requires_grad=True)
    pot = ag.fmm_potential(Xt, Xs, Q, p=12, lmax=3, precision=precision, bbox=(0, 0, 0, 1))
    (pot * torch.tensor(w, device="cuda")).sum().backward()
    # direct references
    dq, _ = oracle.direct(xs, xt, w.astype(np.float32), neq=0, eps2=0.0, exclude_self=True)
    _, gt = oracle.direct(xt, xs, q, neq=0, eps2=0.0, exclude_self=True)
    _, gs = oracle.direct(xs, xt, w.astype(np.float32), neq=0, eps2=0.0, exclude_self=True)
    # w is rounded to float32 on the way into the transposed FMM, like the direct sum above
    assert rel(Q.grad.cpu().numpy(), dq) < 2e-5
    assert rel(Xt.grad.cpu().numpy(), w * gt) < 2e-5
    assert rel(Xs.grad.cpu().numpy(), q * gs) < 2e-5


def test_shared_positions_sum_both_roles(ag, oracle):
    """Targets = sources (one tensor): autograd adds w*grad(pot) and q*grad(psi)."""
    rng = np.random.default_rng(6)
    n = 4000
    x = rng.random((3, n), dtype=np.float32)
    q = rng.standard_normal(n).astype(np.float32)
    w = rng.standard_normal(n).astype(np.float32)
    X = torch.tensor(x, device="cuda", requires_grad=True)
    Q = torch.tensor(q, device="cuda")
    pot = ag.fmm_potential(X, X, Q, p=12, lmax=3, precision=0, bbox=(0, 0, 0, 1))
    (pot * torch.tensor(w, device="cuda")).sum().backward()
    _, g1 = oracle.direct(x, x, q, neq=0, eps2=0.0, exclude_self=True)
    _, g2 = oracle.direct(x, x, w, neq=0, eps2=0.0, exclude_self=True)
    assert rel(X.grad.cpu().numpy(), w * g1 + q * g2) < 2e-5


def test_finite_differences(ag):
    rng = np.random.default_rng(7)
    n = 3000
    x = rng.random((3, n), dtype=np.float32) * 0.9 + 0.05
    q = rng.standard_normal(n).astype(np.float32)
    w = torch.tensor(rng.standard_normal(n), device="cuda")
    X = torch.tensor(x, device="cuda", requires_grad=True)
    Q = torch.tensor(q, device="cuda", dtype=torch.float64, requires_grad=True)
    loss = lambda X_, Q_: (ag.fmm_potential(X_, X_, Q_, p=12, lmax=3, precision=0, bbox=(0, 0, 0, 1)) * w).sum()
    loss(X, Q).backward()
    h = 1e-3
    for _ in range(16):
        d, i = rng.integers(0, 3), rng.integers(0, n)
        xp, xm = x.copy(), x.copy()
        xp[d, i] += h
        xm[d, i] -= h
        with torch.no_grad():
            fd = (loss(torch.tensor(xp, device="cuda"), Q) - loss(torch.tensor(xm, device="cuda"), Q)).item() / (2 * h)
        g = X.grad[d, i].item()
        assert abs(fd - g) <= 1e-2 * max(1.0, abs(g))
    for _ in range(8):
        j = rng.integers(0, n)
        qp, qm = q.astype(np.float64).copy(), q.astype(np.float64).copy()
        qp[j] += 1e-2
        qm[j] -= 1e-2
        with torch.no_grad():
            fd = (loss(X.detach(), torch.tensor(qp, device="cuda")) - loss(X.detach(), torch.tensor(qm, device="cuda"))).item() / 2e-2
        assert abs(fd - Q.grad[j].item()) <= 1e-4 * max(1.0, abs(fd))


@pytest.mark.parametrize("kernel", [1, 2])
def test_normal_kernels_charge_adjoint(kernel, ag, oracle):
    rng = np.random.default_rng(8 + kernel)
    ni, nj = 3000, 3500
    xt = rng.random((3, ni), dtype=np.float32)
    xs = rng.random((3, nj), dtype=np.float32)
    nt = rng.standard_normal((3, ni)).astype(np.float32)
    ns = rng.standard_normal((3, nj)).astype(np.float32)
    q = rng.standard_normal(nj).astype(np.float32)
    w = rng.standard_normal(ni).astype(np.float32)
    Q = torch.tensor(q, device="cuda", requires_grad=True)
    pot = ag.fmm_potential(torch.tensor(xt, device="cuda"), torch.tensor(xs, device="cuda"), Q, kernel=kernel,
                           n_t=torch.tensor(nt, device="cuda"), n_s=torch.tensor(ns, device="cuda"), p=12, lmax=3,
                           precision=0, bbox=(0, 0, 0, 1))
    (pot * torch.tensor(w, device="cuda")).sum().backward()
    # A^T w = -(other normal kernel) with the point sets swapped
    other = 2 if kernel == 1 else 1
    ref, _ = oracle.direct(xs, xt, w, neq=other, eps2=0.0, exclude_self=True,
                           tn=ns if other == 1 else None, sn=nt if other == 2 else None)
    assert rel(Q.grad.cpu().numpy(), -ref) < 2e-5


def gn_direct(xt, nt, xs, ns, q, kernel):
    """FP64 direct sum (numpy, the checker) of the normal-derivative kernels and
    of their gradient w.r.t. the target position with the normals held fixed:
    pot_i = sum_j q_j (d.n)/(4 pi r^3), d = x_i - x_j, n = n_i (Gni) or n_j
    (Gnj); grad_i = sum_j q_j (n/r^3 - 3 (d.n) d / r^5)/(4 pi); zero-distance
    pairs skipped."""
    xt, xs = xt.astype(np.float64), xs.astype(np.float64)
    ni = xt.shape[1]
    pot = np.zeros(ni)
    grad = np.zeros((3, ni))
    for a in range(0, ni, 256):
        b = min(ni, a + 256)
        d = xt[:, a:b, None] - xs[:, None, :]
        r2 = (d * d).sum(0)
        with np.errstate(divide="ignore"):
            ri = np.where(r2 > 0, 1.0 / np.sqrt(np.where(r2 > 0, r2, 1.0)), 0.0)
        n = nt[:, a:b, None].astype(np.float64) if kernel == 1 else ns[:, None, :].astype(np.float64)
        dot = (d * n).sum(0)
        r3 = ri ** 3
        pot[a:b] = (q[None, :] * dot * r3).sum(1)
        grad[:, a:b] = (q[None, None, :] * (n * r3[None] - 3 * dot[None] * r3[None] * ri[None] ** 2 * d)).sum(2)
    return pot / (4 * np.pi), grad / (4 * np.pi)


@pytest.mark.parametrize("kernel", [1, 2])
@pytest.mark.parametrize("precision", [0, 1])
def test_normal_kernels_position_gradients_vs_direct(kernel, precision, ag):
    """Gni / Gnj position gradients through autograd (forward target gradient,
    transposed matvec with its gradient) against the FP64 direct sum:
    dL/dx_t = w grad_t(A q), dL/dx_s = -q sum_i w_i grad_d k(d) = q grad_s(A^T w)."""
    rng = np.random.default_rng(20 + kernel)
    ni, nj = 2000, 2500
    xt = rng.random((3, ni), dtype=np.float32)
    xs = rng.random((3, nj), dtype=np.float32)
    nt = rng.standard_normal((3, ni)).astype(np.float32)
    nt /= np.linalg.norm(nt, axis=0)
    ns = rng.standard_normal((3, nj)).astype(np.float32)
    ns /= np.linalg.norm(ns, axis=0)
    q = rng.standard_normal(nj).astype(np.float32)
    w = rng.standard_normal(ni).astype(np.float32)
    Xt = torch.tensor(xt, device="cuda", requires_grad=True)
    Xs = torch.tensor(xs, device="cuda", requires_grad=True)
    Q = torch.tensor(q, device="cuda", dtype=torch.float64, requires_grad=True)
    pot = ag.fmm_potential(Xt, Xs, Q, kernel=kernel, n_t=torch.tensor(nt, device="cuda"),
                           n_s=torch.tensor(ns, device="cuda"), p=12, lmax=3, precision=precision, bbox=(0, 0, 0, 1))
    (pot * torch.tensor(w, device="cuda", dtype=torch.float64)).sum().backward()
    vd, gt = gn_direct(xt, nt, xs, ns, q.astype(np.float64), kernel)
    assert rel(pot.detach().cpu().numpy(), vd) < 2e-5
    assert rel(Xt.grad.cpu().numpy(), w * gt) < 2e-5
    # source side: d/dx_j of sum_i w_i k(x_i - x_j) = -sum_i w_i grad_d k
    wd = w.astype(np.float64)
    gs = np.zeros((3, nj))
    for a in range(0, nj, 256):
        b = min(nj, a + 256)
        d = xt[:, :, None].astype(np.float64) - xs[:, None, a:b].astype(np.float64)
        r2 = (d * d).sum(0)
        ri = np.where(r2 > 0, 1.0 / np.sqrt(np.where(r2 > 0, r2, 1.0)), 0.0)
        n = nt[:, :, None].astype(np.float64) if kernel == 1 else ns[:, None, a:b].astype(np.float64)
        dot = (d * n).sum(0)
        r3 = ri ** 3
        gs[:, a:b] = -(wd[None, :, None] * (n * r3[None] - 3 * dot[None] * r3[None] * ri[None] ** 2 * d)).sum(1)
    assert rel(Xs.grad.cpu().numpy(), q * gs / (4 * np.pi)) < 2e-5


@pytest.mark.parametrize("kernel", [0, 1, 2])
def test_finite_differences_mixed_clustered(kernel, ag):
    """Central differences (h = 1e-4, 64 random coordinates, each side a fresh
    tree) of L = sum(w * pot) on clustered points (32 Gaussian clusters,
    sigma 0.02: the 1M-point benchmark distribution at 20,000 points), mixed
    form, targets = sources, against the backward's position gradient.  The
    difference quotient itself carries O(h^2 / r^2) truncation (r the moved
    point's nearest-neighbour distance; for the normal-derivative kernels the
    third derivatives grow like r^-5), so the coordinates are drawn among
    points with no neighbour closer than 30 h; with the FP32 rounding of the
    near field that leaves a few 1e-3, hence the 1e-2 bound on the 2-norm
    relative error.  (The exact check is against the FP64 direct sums.)"""
    rng = np.random.default_rng(40 + kernel)
    n, ncl = 20000, 32
    c = rng.uniform(0.1, 0.9, (3, ncl))
    x = np.clip(c[:, rng.integers(0, ncl, n)] + 0.02 * rng.standard_normal((3, n)), 0.0, 1.0).astype(np.float32)
    nr = rng.standard_normal((3, n)).astype(np.float32)
    nr /= np.linalg.norm(nr, axis=0)
    q = rng.standard_normal(n).astype(np.float32)
    w = torch.tensor(rng.standard_normal(n), device="cuda")
    nd = torch.tensor(nr, device="cuda")
    Q = torch.tensor(q, device="cuda", dtype=torch.float64)

    def loss(X_):
        return (ag.fmm_potential(X_, X_, Q, kernel=kernel, n_t=nd, n_s=nd, p=12, lmax=4, precision=1,
                                 bbox=(0, 0, 0, 1)) * w).sum()

    X = torch.tensor(x, device="cuda", requires_grad=True)
    loss(X).backward()
    an = X.grad.cpu().numpy()
    h = 1e-4
    fd, ref = [], []
    x64 = x.astype(np.float64)
    while len(fd) < 64:
        d, i = int(rng.integers(0, 3)), int(rng.integers(0, n))
        r2 = ((x64 - x64[:, i:i + 1]) ** 2).sum(0)
        r2[i] = np.inf
        if r2.min() < (30 * h) ** 2:
            continue
        xp, xm = x.copy(), x.copy()
        xp[d, i] = np.float32(x[d, i] + h)
        xm[d, i] = np.float32(x[d, i] - h)
        with torch.no_grad():
            lp = loss(torch.tensor(xp, device="cuda")).item()
            lm = loss(torch.tensor(xm, device="cuda")).item()
        fd.append((lp - lm) / (float(xp[d, i]) - float(xm[d, i])))
        ref.append(an[d, i])
    assert rel(fd, ref) < 1e-2
