"""fmmb_evaluate_transpose and fmmb_position_grad (the adjoint entry points)
against the oracle's FP64 direct sums, through the C ABI.

A is the plan's matvec pot_i = sum_j K(x_i, x_j) q_j.  Its transpose:
  G   (symmetric):          A^T w = G(targets = x_s, sources = x_t, charges w)
  Gni (target normals n_t): A^T w = -Gnj(targets = x_s, sources = x_t with n_t)
  Gnj (source normals n_s): A^T w = -Gni(targets = x_s with n_s, sources = x_t)
since d/dx_j G(x_i - x_j) = -d/dx_i G(x_i - x_j).  Position gradients of
L = sum_i w_i pot_i (G only): dL/dx_t = w * grad pot(x_t),
dL/dx_s = q * grad psi(x_s) with psi = A^T w.
Tolerances: 2e-5 relative at p = 12 (FMM truncation ~1e-6 on potentials, a few
1e-6 on fields), and the transposed plan must reproduce a plan built directly on
the swapped sets to 1e-12 (same trees, same arithmetic).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def ob():
    import old_fmm_bem_b200 as ob
    from old_fmm_bem_b200 import build
    build.build()
    return ob


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _sets(seed, ni, nj):
    rng = np.random.default_rng(seed)
    xt = rng.random((3, ni), dtype=np.float32)
    xs = rng.random((3, nj), dtype=np.float32)
    nt = rng.standard_normal((3, ni)).astype(np.float32)
    ns = rng.standard_normal((3, nj)).astype(np.float32)
    q = rng.standard_normal(nj).astype(np.float32)
    w = rng.standard_normal(ni).astype(np.float32)
    return xt, xs, nt, ns, q, w


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("kernel", [0, 1, 2])
def test_transpose_vs_direct(kernel, precision, ob, oracle):
    xt, xs, nt, ns, q, w = _sets(20 + kernel, 3000, 4500)
    pl = ob.Plan(kernel=kernel, p=12, lmax=3, precision=precision, semantics=1, exclude_self=True)
    pl.set_geometry(xt, xs, nt if kernel == 1 else None, ns if kernel == 2 else None, bbox=(0, 0, 0, 1))
    out, grad = pl.evaluate_transpose(w, f64=True)
    assert out.shape == (4500,)
    if kernel == 0:
        ref, gref = oracle.direct(xs, xt, w, neq=0, eps2=0.0, exclude_self=True)
        assert rel(out, ref) < 2e-5
        assert rel(grad.reshape(3, -1), gref) < 2e-5
    else:
        other = 2 if kernel == 1 else 1
        ref, _ = oracle.direct(xs, xt, w, neq=other, eps2=0.0, exclude_self=True,
                               tn=ns if other == 1 else None, sn=nt if other == 2 else None)
        assert grad is None
        assert rel(out, -ref) < 2e-5
    # the forward still works after the transposed plan was built, on the same trees
    pot, _ = pl.evaluate(q, f64=True)
    ref_f, _ = oracle.direct(xt, xs, q, neq=kernel, eps2=0.0, exclude_self=True,
                             tn=nt if kernel == 1 else None, sn=ns if kernel == 2 else None)
    assert rel(pot, ref_f) < 2e-5
    pl.close()


def test_transpose_equals_swapped_plan(ob):
    """The transposed plan is a plan on the swapped sets with the same box:
    its result equals that of a plan built by hand (G kernel, FP32 outputs,
    device buffers, then a second call reusing the transposed plan)."""
    xt, xs, nt, ns, q, w = _sets(30, 5000, 3000)
    pl = ob.Plan(kernel=0, p=10, lmax=3, precision=1, semantics=1, exclude_self=True)
    pl.set_geometry(xt, xs, bbox=(0, 0, 0, 1))
    W = torch.from_numpy(w).cuda()
    out = torch.zeros(3000, device="cuda")
    grad = torch.zeros(9000, device="cuda")
    pl.evaluate_transpose(W, out, grad)
    torch.cuda.synchronize()
    ps = ob.Plan(kernel=0, p=10, lmax=3, precision=1, semantics=1, exclude_self=True)
    ps.set_geometry(xs, xt, bbox=(0, 0, 0, 1))
    ref, gref = ps.evaluate(w)
    assert rel(out.cpu().numpy(), ref) < 1e-6
    assert rel(grad.cpu().numpy(), gref) < 1e-6
    # second call: same plan, new weights
    w2 = (w * 0.5 + 1.0).astype(np.float32)
    o2, _ = pl.evaluate_transpose(w2)
    r2, _ = ps.evaluate(w2)
    assert rel(o2, r2) < 1e-6
    pl.close()
    ps.close()


def test_position_grad_vs_direct(ob, oracle):
    xt, xs, nt, ns, q, w = _sets(40, 3500, 4000)
    pl = ob.Plan(kernel=0, p=12, lmax=3, precision=1, semantics=1, exclude_self=True)
    pl.set_geometry(xt, xs, bbox=(0, 0, 0, 1))
    dxt, dxs = pl.position_grad(q, w)
    _, gt = oracle.direct(xt, xs, q, neq=0, eps2=0.0, exclude_self=True)
    _, gs = oracle.direct(xs, xt, w, neq=0, eps2=0.0, exclude_self=True)
    assert rel(dxt, w.astype(np.float64) * gt) < 2e-5
    assert rel(dxs, q.astype(np.float64) * gs) < 2e-5
    # device outputs give the same numbers
    Dt = torch.zeros(3 * 3500, dtype=torch.float64, device="cuda")
    Ds = torch.zeros(3 * 4000, dtype=torch.float64, device="cuda")
    pl.position_grad(torch.from_numpy(q).cuda(), torch.from_numpy(w).cuda(), Dt, Ds)
    torch.cuda.synchronize()
    assert rel(Dt.cpu().numpy(), dxt.ravel()) < 1e-9
    assert rel(Ds.cpu().numpy(), dxs.ravel()) < 1e-9
    pl.close()


def test_position_grad_rejects_normal_kernels(ob):
    xt, xs, nt, ns, q, w = _sets(50, 500, 500)
    pl = ob.Plan(kernel=2, p=6, lmax=2)
    pl.set_geometry(xt, xs, None, ns, bbox=(0, 0, 0, 1))
    with pytest.raises(ob.FMMError):
        pl.position_grad(q, w)
    pl.close()


@pytest.mark.parametrize("shared", [False, True])
def test_adjoint_host_buffers(shared, ob, oracle):
    """fmmb_adjoint_f64 with host charges, weights and outputs (its copies of
    q to the device and of dL/dx_t to the host overlap the transposed matvec
    on a second stream) gives the numbers of the device-buffer call, and both
    match the direct sums; the forward field is given on the device (as the
    forward leaves it) and on the host."""
    xt, xs, nt, ns, q, w = _sets(60, 3200, 3200 if shared else 4100)
    if shared:
        xs = xt
    ni, nj = xt.shape[1], xs.shape[1]
    pl = ob.Plan(kernel=0, p=12, lmax=3, precision=1, semantics=1, exclude_self=True)
    pl.set_geometry(xt, xs, bbox=(0, 0, 0, 1))
    pot, field = pl.evaluate(q, f64=True)
    field = np.ascontiguousarray(field, np.float64).reshape(-1)
    _, gt = oracle.direct(xt, xs, q, neq=0, eps2=0.0, exclude_self=True)
    aw, gs = oracle.direct(xs, xt, w, neq=0, eps2=0.0, exclude_self=True)
    for fld in (field, torch.from_numpy(field).cuda()):
        for _ in range(2):  # a second call reuses the copy stream and the staged buffers
            dq, dxt, dxs = pl.adjoint(q, w, fld, want_dxs=True)
            assert rel(dq, aw) < 2e-5
            assert rel(dxt.reshape(3, -1), w.astype(np.float64) * gt) < 2e-5
            assert rel(dxs.reshape(3, -1), q.astype(np.float64) * gs) < 2e-5
    Dq = torch.zeros(nj, dtype=torch.float64, device="cuda")
    Dt = torch.zeros(3 * ni, dtype=torch.float64, device="cuda")
    Ds = torch.zeros(3 * nj, dtype=torch.float64, device="cuda")
    pl.adjoint(torch.from_numpy(q).cuda(), torch.from_numpy(w).cuda(), torch.from_numpy(field).cuda(), Dq, Dt, Ds,
               want_dxs=True)
    torch.cuda.synchronize()
    # (the upward pass adds children into parents with FP64 atomics in no fixed
    # order, and an ulp of a multipole can move a rounding of the FP32 tensor-core
    # M2L: runs agree to ~1e-10, as the position-gradient test allows)
    assert rel(Dq.cpu().numpy(), dq) < 1e-9
    assert rel(Dt.cpu().numpy(), dxt) < 1e-9
    assert rel(Ds.cpu().numpy(), dxs) < 1e-9
    pl.close()
