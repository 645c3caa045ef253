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
