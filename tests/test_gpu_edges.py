"""Edge cases of the plan API on the GPU, against the oracle's FP64 direct sum:
a single target and source, every point at one position (zero distances only),
points on the far faces of the root cube (clamped into the last box like the
reference's boxn), the shallowest and the deepest octree, more targets than
sources and the reverse, and ragged problem sizes in a forest.  Tolerance:
1e-6 relative at p = 12 (FMM truncation; 3e-6 with points on the root's far
faces, where the expansions about the last boxes converge slowest, and 5e-5
for the gradient at depth 8, while the same algorithm restated on the CPU
agrees to 1e-10), exact zeros where every pair is excluded."""
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
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _plan(ob, kernel=0, lmax=3, p=12, precision=0):
    return ob.Plan(kernel=kernel, p=p, lmax=lmax, precision=precision, semantics=1, exclude_self=True)


@pytest.mark.parametrize("precision", [0, 1])
def test_single_point_pair(precision, ob, oracle):
    t = np.array([[0.2], [0.3], [0.4]], np.float32)
    s = np.array([[0.7], [0.6], [0.1]], np.float32)
    q = np.array([0.5], np.float32)
    pl = _plan(ob, precision=precision)
    pl.set_geometry(t, s, bbox=(0, 0, 0, 1))
    v, g = pl.evaluate(q, f64=True)
    ref, gref = oracle.direct(t, s, q, neq=0, eps2=0.0, exclude_self=True)
    assert rel(v, ref) < 1e-6 and rel(g.reshape(3, -1), gref) < 1e-6
    pl.close()


def test_all_points_coincident(ob):
    x = np.full((3, 500), 0.37, np.float32)
    q = np.random.default_rng(1).uniform(-1, 1, 500).astype(np.float32)
    for kernel in (0, 1, 2):
        pl = _plan(ob, kernel=kernel)
        nrm = np.ones((3, 500), np.float32)
        pl.set_geometry(x, x, nrm if kernel == 1 else None, nrm if kernel == 2 else None, bbox=(0, 0, 0, 1))
        v, g = pl.evaluate(q, f64=True)
        assert np.all(v == 0.0)
        if g is not None:
            assert np.all(g == 0.0)
        pl.close()


@pytest.mark.parametrize("lmax", [2, 8])
def test_points_on_the_far_faces_and_depths(lmax, ob, oracle):
    rng = np.random.default_rng(2 + lmax)
    n = 4000
    x = rng.random((3, n), dtype=np.float32)
    x[0, :200] = 1.0  # on the far face x = xmin + rd: clamped into the last box
    x[1, 200:400] = 1.0
    x[2, 400:600] = 1.0
    x[:, 600:610] = 1.0  # the far corner
    q = rng.uniform(-1, 1, n).astype(np.float32)
    pl = _plan(ob, lmax=lmax)
    pl.set_geometry(x, x, bbox=(0, 0, 0, 1))
    v, g = pl.evaluate(q, f64=True)
    # the same algorithm on the CPU (oracle restatement, FP64, same depth and order): 1e-10
    vo, go = oracle.oracle_fmm(x, x, q, neq=0, p=12, lmax=lmax, ref_semantics=False, eps2=0.0, exclude_self=True)
    assert rel(v, vo) < 1e-10 and rel(g.reshape(3, -1), go) < 1e-10
    # against the direct sum: truncation, larger for the gradient and for deep trees (more M2L levels)
    ref, gref = oracle.direct(x, x, q, neq=0, eps2=0.0, exclude_self=True, targets=(0, 1000))
    assert rel(v[:1000], ref) < 3e-6
    assert rel(g.reshape(3, -1)[:, :1000], gref) < 5e-5
    pl.close()


@pytest.mark.parametrize("ni,nj", [(7, 20000), (20000, 7)])
def test_unbalanced_sets(ni, nj, ob, oracle):
    rng = np.random.default_rng(ni)
    t = rng.random((3, ni), dtype=np.float32)
    s = rng.random((3, nj), dtype=np.float32)
    sn = rng.standard_normal((3, nj)).astype(np.float32)
    q = rng.uniform(-1, 1, nj).astype(np.float32)
    pl = _plan(ob, kernel=2, lmax=4)
    pl.set_geometry(t, s, None, sn, bbox=(0, 0, 0, 1))
    v, _ = pl.evaluate(q, f64=True)
    vo, _ = oracle.oracle_fmm(t, s, q, neq=2, p=12, lmax=4, sn=sn, ref_semantics=False, eps2=0.0,
                              exclude_self=True)
    assert rel(v, vo) < 1e-10
    m = min(ni, 1000)
    ref, _ = oracle.direct(t, s, q, neq=2, eps2=0.0, exclude_self=True, sn=sn, targets=(0, m))
    assert rel(v[:m], ref) < 1e-5  # the double-layer kernel truncates slower than G at p = 12
    pl.close()


def test_ragged_forest(ob, oracle):
    """Problems of 1, 2, 3000 and 17 points (and an empty one) in one plan,
    mixed form (FP32 near field: 2e-6)."""
    rng = np.random.default_rng(9)
    sizes = [1, 2, 0, 3000, 17]
    xs = [rng.random((3, n), dtype=np.float32) for n in sizes]
    off = np.cumsum([0] + sizes).astype(np.int32)
    x = np.ascontiguousarray(np.concatenate(xs, axis=1))
    q = rng.uniform(-1, 1, x.shape[1]).astype(np.float32)
    pl = _plan(ob, lmax=4, precision=1)
    pl.set_geometry_batch(off, x, off, x, bbox=(0, 0, 0, 1))
    v, _ = pl.evaluate(q, f64=True)
    pl.close()
    for b, n in enumerate(sizes):
        if n == 0:
            continue
        ref, _ = oracle.direct(xs[b], xs[b], q[off[b]:off[b + 1]], neq=0, eps2=0.0, exclude_self=True)
        if n == 1:
            assert v[off[b]] == 0.0
        else:
            assert rel(v[off[b]:off[b + 1]], ref) < 2e-6  # mixed form
