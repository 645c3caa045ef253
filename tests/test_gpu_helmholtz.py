"""The complex Helmholtz kernel e^{ikr}/(4 pi r) (FMMB_HELMHOLTZ_G) through the
C ABI, against the FP64 complex direct sum of oracle/helmholtz_oracle.py.

Parity is unpinned (the reference has no oscillatory Helmholtz kernel): the
checks are the kernel's definition, convergence in p, the k -> 0 limit against
the pinned Laplace G path, and the transpose.  Tolerances:
* GPU direct sum vs numpy direct: 1e-12;
* FMM in FP64 at p = 16 vs direct: 1e-6 (truncation of the expansions);
* mixed form (FP32 P2P) vs FP64 form: 2e-6;
* k = 1e-3: Re(phi) equals the Laplace G potential to 1e-5, Im(phi) equals
  k/(4 pi) sum q to 1e-5 (the O((kr)^2) terms).
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
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


BOX = (-1.0001, -1.0001, -1.0001, 2.0002)


def _plan(ob, p, lmax, precision=0, k=5.0, nrhs=1):
    return ob.Plan(kernel=ob.HELMHOLTZ_G, p=p, lmax=lmax, precision=precision, semantics=1, exclude_self=True,
                   wavenumber=k, nrhs=nrhs)


def test_direct_matches_numpy(ob):
    from oracle import helmholtz_oracle as ho
    x, q = ho.sphere_points(3000, 1)
    y, _ = ho.sphere_points(2000, 2)
    pl = _plan(ob, 4, 2)
    pl.set_geometry(y, x, bbox=BOX)
    v, _ = pl.direct(q, 0, 2000)
    pl.close()
    assert rel(v, ho.direct(y, x, q, 5.0)) < 1e-12


@pytest.mark.parametrize("lmax", [3, 4])
def test_fmm_fp64_vs_direct_and_convergence(lmax, ob):
    from oracle import helmholtz_oracle as ho
    x, q = ho.sphere_points(20000, 3 + lmax)
    ref = ho.direct(x[:, :1500], x, q, 5.0)
    errs = {}
    for p in (6, 10, 16):
        pl = _plan(ob, p, lmax)
        pl.set_geometry(x, x, bbox=BOX)
        v, _ = pl.evaluate(q, f64=True)
        pl.close()
        errs[p] = rel(v[:1500], ref)
    assert errs[16] < 1e-6, errs
    assert errs[6] > errs[10] > errs[16], errs


def test_mixed_matches_fp64_and_nrhs(ob):
    from oracle import helmholtz_oracle as ho
    x, q = ho.sphere_points(15000, 9)
    q2 = np.concatenate([q, (q * 2j).astype(np.complex64)])  # exact in complex64
    out = []
    for prec in (0, 1):
        pl = _plan(ob, 12, 3, precision=prec, nrhs=2)
        pl.set_geometry(x, x, bbox=BOX)
        v, _ = pl.evaluate(q2, f64=True)
        pl.close()
        out.append(v)
    assert rel(out[1], out[0]) < 2e-6
    # the second right-hand side is the first times 2i
    assert rel(out[0][15000:], out[0][:15000] * 2j) < 1e-12


def test_low_frequency_limit_is_laplace(ob):
    from oracle import helmholtz_oracle as ho
    x, qc = ho.sphere_points(12000, 11)
    q = qc.real.astype(np.float32)
    k = 1e-3
    pl = _plan(ob, 10, 3, k=k)
    pl.set_geometry(x, x, bbox=BOX)
    v, _ = pl.evaluate(q.astype(np.complex64), f64=True)
    pl.close()
    lp = ob.Plan(kernel=ob.LAPLACE_G, p=10, lmax=3, precision=0, semantics=1, exclude_self=True)
    lp.set_geometry(x, x, bbox=BOX)
    vl, _ = lp.evaluate(q, f64=True)
    lp.close()
    assert rel(v.real, vl) < 1e-5
    qsum = q.astype(np.float64).sum() - q.astype(np.float64)  # self pairs excluded
    assert rel(v.imag, k / (4 * np.pi) * qsum) < 1e-5


def test_transpose_and_forest(ob):
    from oracle import helmholtz_oracle as ho
    xt, w = ho.sphere_points(6000, 13)
    xs, _ = ho.sphere_points(9000, 14)
    xs = (0.8 * xs).astype(np.float32)
    pl = _plan(ob, 14, 3)
    pl.set_geometry(xt, xs, bbox=BOX)
    out, _ = pl.evaluate_transpose(w, f64=True)  # A^T w: targets xs, sources xt
    pl.close()
    assert rel(out, ho.direct(xs, xt, w, 5.0)) < 1e-6
    # two independent problems in one plan
    t_off = np.array([0, 6000, 6000 + 9000], np.int32)
    x = np.ascontiguousarray(np.concatenate([xt, xs], axis=1))
    q = np.concatenate([w, w[:9000 - 6000], w]).astype(np.complex64)[:15000]
    pf = _plan(ob, 14, 3)
    pf.set_geometry_batch(t_off, x, t_off, x, bbox=BOX)
    v, _ = pf.evaluate(q, f64=True)
    pf.close()
    assert rel(v[:6000], ho.direct(xt, xt, q[:6000], 5.0)) < 1e-6
    assert rel(v[6000:], ho.direct(xs, xs, q[6000:], 5.0)) < 1e-6


@pytest.mark.parametrize("precision", [0, 1])
def test_yukawa_fmm_vs_direct(precision, ob):
    """FMMB_YUKAWA (the reference's neq 10 kernel, (pi/2) e^{-l r}/(l r)) in
    accurate semantics: GPU direct sum = numpy to 1e-12; FMM at p = 14 within
    1e-6 (FP64) / 2e-6 (mixed), the error shrinking from p = 6 to 10 to 14."""
    from oracle import helmholtz_oracle as ho
    rng = np.random.default_rng(31)
    x = rng.random((3, 20000), dtype=np.float32)
    q = rng.uniform(-1, 1, 20000).astype(np.float32)
    lam = 4.0
    ref = ho.yukawa_direct(x[:, :1500], x, q, lam)
    errs = {}
    for p in (6, 10, 14):
        pl = ob.Plan(kernel=ob.YUKAWA, p=p, lmax=4, precision=precision, semantics=1, exclude_self=True,
                     wavenumber=lam)
        pl.set_geometry(x, x, bbox=(0, 0, 0, 1))
        v, g = pl.evaluate(q, f64=True)
        assert g is None
        if p == 14:
            d, _ = pl.direct(q, 0, 1500)
            assert rel(d, ref) < 1e-12
        pl.close()
        errs[p] = rel(v[:1500], ref)
    assert errs[14] < (1e-6 if precision == 0 else 2e-6), errs
    assert errs[6] > errs[10] > errs[14], errs
