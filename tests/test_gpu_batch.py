"""Many independent problems in one plan (fmmb_set_geometry_batch) and the
batched device GMRES (fmmb_gmres), through the C ABI.

Tolerances:
* forest plan vs one plan per problem over the same root cube and depth: the
  same boxes, lists and operators, so 1e-12 relative in FP64 (only the order
  of M2M atomics differs) and 1e-6 in the mixed form (the tensor-core M2L
  groups pairs of all problems into shared tiles);
* forest direct sum vs the oracle's FP64 direct sum per problem: 1e-12;
* GMRES vs the numpy GMRES of oracle/bem_oracle.py on the dense operator, same
  iteration count: 50 x the FMM's own matvec error on the same problem (the
  iterates are continuous in the operator; the systems are well conditioned,
  cond ~ 1.7), and vs numpy.linalg.solve after convergence likewise.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


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


def _clustered(rng, n, centre):
    return np.clip(centre[:, None] + 0.08 * rng.standard_normal((3, n)), 0, 1).astype(np.float32)


def _problems(seed, sizes):
    rng = np.random.default_rng(seed)
    out = []
    for n in sizes:
        c = rng.random(3)
        t = _clustered(rng, n, c)
        s = _clustered(rng, n + 17, c)
        tn = rng.standard_normal((3, n)).astype(np.float32)
        sn = rng.standard_normal((3, n + 17)).astype(np.float32)
        out.append((t, tn, s, sn))
    return out


def _concat(probs):
    t_off = np.cumsum([0] + [p[0].shape[1] for p in probs])
    s_off = np.cumsum([0] + [p[2].shape[1] for p in probs])
    cat = [np.ascontiguousarray(np.concatenate([p[k] for p in probs], axis=1)) for k in range(4)]
    return t_off, s_off, cat


@pytest.mark.parametrize("kernel", [0, 1, 2])
@pytest.mark.parametrize("precision", [0, 1])
def test_forest_equals_one_plan_per_problem(kernel, precision, ob):
    probs = _problems(10 + kernel, [4000, 0, 9000, 2500, 6000])
    t_off, s_off, (t, tn, s, sn) = _concat(probs)
    nrhs = 2
    rng = np.random.default_rng(5)
    q = rng.uniform(-1, 1, nrhs * s.shape[1]).astype(np.float32)
    kw = dict(kernel=kernel, p=10, lmax=4, precision=precision, semantics=1, exclude_self=True, nrhs=nrhs)
    bbox = (0, 0, 0, 1)
    pl = ob.Plan(**kw)
    pl.set_geometry_batch(t_off, t, s_off, s, tn if kernel == 1 else None, sn if kernel == 2 else None, bbox=bbox)
    pot, grad = pl.evaluate(q, f64=True)
    pl.close()
    nt, ns = t.shape[1], s.shape[1]
    tol = 1e-12 if precision == 0 else 1e-6
    for b, (pt, ptn, ps, psn) in enumerate(probs):
        if pt.shape[1] == 0:
            continue
        one = ob.Plan(**kw)
        one.set_geometry(pt, ps, ptn if kernel == 1 else None, psn if kernel == 2 else None, bbox=bbox)
        qb = np.concatenate([q[r * ns + s_off[b]:r * ns + s_off[b + 1]] for r in range(nrhs)])
        pb, gb = one.evaluate(qb, f64=True)
        one.close()
        mine = np.concatenate([pot[r * nt + t_off[b]:r * nt + t_off[b + 1]] for r in range(nrhs)])
        assert rel(mine, pb) < tol, b
        if kernel == 0:
            g = grad.reshape(nrhs, 3, nt)
            mg = np.concatenate([g[r][:, t_off[b]:t_off[b + 1]].ravel() for r in range(nrhs)])
            assert rel(mg, gb) < tol * 10, b


def test_forest_direct_sum_per_problem(ob, oracle):
    probs = _problems(20, [3000, 5000, 1200])
    t_off, s_off, (t, tn, s, sn) = _concat(probs)
    q = np.random.default_rng(6).uniform(-1, 1, s.shape[1]).astype(np.float32)
    pl = ob.Plan(kernel=0, p=6, lmax=3, semantics=1, exclude_self=True)
    pl.set_geometry_batch(t_off, t, s_off, s, bbox=(0, 0, 0, 1))
    v, g = pl.direct(q, 1000, 8500)  # spans all three problems
    pl.close()
    for b, (pt, _, ps, _) in enumerate(probs):
        a0, a1 = max(1000, t_off[b]), min(8500, t_off[b + 1])
        if a0 >= a1:
            continue
        ref, gref = oracle.direct(pt, ps, q[s_off[b]:s_off[b + 1]], neq=0, eps2=0.0, exclude_self=True,
                                  targets=(a0 - t_off[b], a1 - t_off[b]))
        assert rel(v[a0 - 1000:a1 - 1000], ref) < 1e-12
        assert rel(g[:, a0 - 1000:a1 - 1000], gref) < 1e-12


def _bem_batch(freqs):
    from old_fmm_bem_b200 import geometry
    out = []
    for f in freqs:
        v, fc = geometry.geodesic_sphere(f)
        x, n, w, _ = geometry.quadrature_points(v, fc, "centroid")
        out.append((x, n, w))
    return out


@pytest.mark.parametrize("kernel", [1, 2])
def test_gmres_matches_numpy_gmres(kernel, ob):
    from old_fmm_bem_b200 import geometry
    from oracle import bem_oracle
    probs = _bem_batch([5, 8, 11])
    off = np.cumsum([0] + [p[0].shape[1] for p in probs])
    x = np.ascontiguousarray(np.concatenate([p[0] for p in probs], axis=1))
    nrm = np.ascontiguousarray(np.concatenate([p[1] for p in probs], axis=1))
    area = np.concatenate([p[2] for p in probs])
    n, nrhs = x.shape[1], 2
    weight = (area / geometry.E1).astype(np.float32)
    rng = np.random.default_rng(kernel)
    b = rng.uniform(-1, 1, nrhs * n)
    pl = ob.Plan(kernel=kernel, p=14, lmax=3, precision=0, semantics=1, exclude_self=True, nrhs=nrhs)
    pl.set_geometry_batch(off, x, off, x, nrm if kernel == 1 else None, nrm if kernel == 2 else None,
                          bbox=(-1.01, -1.01, -1.01, 2.02))
    iters = 6
    xs, it, resid = pl.gmres(b, weight=weight, diag=geometry.BEM_DIAG, precond=1 / geometry.BEM_DIAG, restart=4,
                             max_iter=iters)
    assert it == iters and resid.shape == (nrhs, 3)
    # FMM matvec error on these problems (the scale of the allowed difference)
    qv = (weight * rng.uniform(-1, 1, n)).astype(np.float32)
    pl1 = ob.Plan(kernel=kernel, p=14, lmax=3, precision=0, semantics=1, exclude_self=True)
    pl1.set_geometry_batch(off, x, off, x, nrm if kernel == 1 else None, nrm if kernel == 2 else None,
                           bbox=(-1.01, -1.01, -1.01, 2.02))
    fm, _ = pl1.evaluate(qv, f64=True)
    pl1.close()
    efmm = max(1e-10, max(rel(fm[off[k]:off[k + 1]],
                              bem_oracle.kernel_matrix(probs[k][0], kernel, nt=probs[k][1], ns=probs[k][1])
                              @ qv[off[k]:off[k + 1]].astype(np.float64)) for k in range(3)))
    for k in range(3):
        A = bem_oracle.bem_matrix(probs[k][0], probs[k][1], weight[off[k]:off[k + 1]], kernel, geometry.BEM_DIAG)
        for r in range(nrhs):
            bk = b[r * n + off[k]:r * n + off[k + 1]]
            xr, itr, relr = bem_oracle.gmres(A, bk, precond=1 / geometry.BEM_DIAG, restart=4, max_iter=iters)
            mine = xs[r * n + off[k]:r * n + off[k + 1]]
            assert rel(mine, xr) < 50 * efmm, (k, r, rel(mine, xr), efmm)
            assert abs(resid[r, k] - relr) <= 0.05 * relr + 50 * efmm
    # to convergence, against the dense solve
    xs, it, resid = pl.gmres(b, weight=weight, diag=geometry.BEM_DIAG, precond=1 / geometry.BEM_DIAG, restart=8,
                             max_iter=60, rtol=1e-11)
    # resid is the residual of the returned x through the FMM (not the Givens
    # estimate that stopped the iteration at 1e-11): finite-precision GMRES
    # attains 1e-10 .. 2e-9 on these systems
    assert it < 60 and np.all(resid <= 1e-8)
    for k in range(3):
        A = bem_oracle.bem_matrix(probs[k][0], probs[k][1], weight[off[k]:off[k + 1]], kernel, geometry.BEM_DIAG)
        for r in range(nrhs):
            sol = np.linalg.solve(A, b[r * n + off[k]:r * n + off[k + 1]])
            assert rel(xs[r * n + off[k]:r * n + off[k + 1]], sol) < 50 * efmm
    pl.close()


def test_gmres_device_arrays_and_mixed(ob):
    """Device (torch) inputs and the mixed form: the same solution to the
    mixed form's matvec error."""
    torch = pytest.importorskip("torch")
    from old_fmm_bem_b200 import geometry
    probs = _bem_batch([9, 13])
    off = np.cumsum([0] + [p[0].shape[1] for p in probs])
    x = np.ascontiguousarray(np.concatenate([p[0] for p in probs], axis=1))
    nrm = np.ascontiguousarray(np.concatenate([p[1] for p in probs], axis=1))
    weight = (np.concatenate([p[2] for p in probs]) / geometry.E1).astype(np.float32)
    b = np.random.default_rng(9).uniform(-1, 1, x.shape[1])
    out = []
    for prec in (0, 1):
        pl = ob.Plan(kernel=1, p=10, lmax=3, precision=prec, semantics=1, exclude_self=True)
        pl.set_geometry_batch(off, torch.from_numpy(x).cuda(), off, torch.from_numpy(x).cuda(),
                              torch.from_numpy(nrm).cuda(), None, bbox=(-1.01, -1.01, -1.01, 2.02))
        X = torch.zeros(x.shape[1], dtype=torch.float64, device="cuda")
        pl.gmres(torch.from_numpy(b).cuda(), X, torch.from_numpy(weight).cuda(), diag=geometry.BEM_DIAG,
                 precond=1 / geometry.BEM_DIAG, max_iter=12)
        torch.cuda.synchronize()
        out.append(X.cpu().numpy())
        pl.close()
    assert rel(out[1], out[0]) < 1e-5
