"""GPU parity of libfmmb against the oracle (restatement pinned to the
reference) and the reference's golden vectors, through the C ABI.

Tolerances:
* tree, permutations, leaf ranges, lists: bit-exact;
* expansions and potentials, FP64 form vs oracle on the same semantics:
  1e-10 relative (rounding order only);
* FP64 form vs the reference's own float outputs (golden): 1e-6 relative
  (the reference accumulates its outputs in float);
* accuracy vs the FP64 direct sum (accurate semantics): the FMM truncation
  error of the order used, stated per test.
"""
import glob
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "ref_fmm_*.npz")))


@pytest.fixture(scope="module")
def ob():
    import old_fmm_bem_b200 as ob
    from old_fmm_bem_b200 import build
    build.build()
    return ob


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm(a.astype(np.result_type(a, b, np.float64)) - b) / np.linalg.norm(b))


def make_points(n, seed, kind="uniform"):
    rng = np.random.default_rng(seed)
    if kind == "uniform":
        t = rng.random((3, n), dtype=np.float32)
        s = rng.random((3, n), dtype=np.float32)
    else:  # clustered: uneven leaves and empty boxes
        c = rng.random((3, 8))
        t = np.clip(c[:, rng.integers(0, 8, n)] + 0.06 * rng.standard_normal((3, n)), 0, 1).astype(np.float32)
        s = np.clip(c[:, rng.integers(0, 8, n)] + 0.06 * rng.standard_normal((3, n)), 0, 1).astype(np.float32)
    tn = rng.standard_normal((3, n)).astype(np.float32)
    tn /= np.linalg.norm(tn, axis=0)
    sn = rng.standard_normal((3, n)).astype(np.float32)
    sn /= np.linalg.norm(sn, axis=0)
    q = rng.uniform(-1, 1, n).astype(np.float32)
    return t, tn, s, sn, q


def plan_for(ob, neq, p, lmax, t, tn, s, sn, bbox=(0, 0, 0, 1), **kw):
    pl = ob.Plan(kernel=neq, p=p, lmax=lmax, **kw)
    pl.set_geometry(t, s, tn if neq == 1 else None, sn if neq == 2 else None, bbox=bbox)
    return pl


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_tree_and_potentials_match_reference_golden(path, ob, oracle):
    d = np.load(path)
    p, lmax = int(d["p"]), int(d["lmax"])
    for neq in (0, 1, 2):
        pl = plan_for(ob, neq, p, lmax, d["t"], d["tn"], d["s"], d["sn"])
        if neq == 0:
            assert np.array_equal(pl.tree(0), d["perm_i"])
            assert np.array_equal(pl.tree(1), d["perm_j"])
            assert np.array_equal(pl.tree(6), d["leaf_i"])
            assert np.array_equal(pl.tree(7), d["leaf_j"])
            la, lb = oracle.parse_lists(pl.tree(8)), oracle.parse_lists(d["lists"])
            assert len(la) == len(lb)
            for x, y in zip(la, lb):
                assert x[0] == y[0] and x[1] == y[1] and x[3] == y[3]
        v, g = pl.evaluate(d["q"], f64=True)
        ref = d[f"v{neq}"].astype(np.float64)
        assert rel(v, ref) < 1e-6
        if neq == 0:
            assert rel(g.reshape(3, -1), d["g0"]) < 1e-6
        pl.close()


@pytest.mark.parametrize("kind", ["uniform", "clustered"])
@pytest.mark.parametrize("lmax", [2, 3, 4])
def test_tree_bit_exact_vs_oracle(kind, lmax, ob, oracle):
    t, tn, s, sn, q = make_points(6000 if lmax < 4 else 20000, 30 + lmax, kind)
    pl = plan_for(ob, 0, 4, lmax, t, tn, s, sn)
    oracle.oracle_fmm(t, s, q, neq=0, p=4, lmax=lmax)
    rec = oracle.oracle_records()
    for k in (0, 1, 2, 3, 4, 5, 6, 7, 8):
        assert np.array_equal(pl.tree(k), rec[k]), k
    pl.close()


@pytest.mark.parametrize("neq", [0, 1, 2])
@pytest.mark.parametrize("semantics", [0, 1])
def test_fp64_expansions_and_potential_vs_oracle(neq, semantics, ob, oracle):
    """Per-operator parity: multipoles (P2P/P2M/M2M) and locals (M2L/L2L) of
    every level, then the potentials, FP64 form vs the restated reference."""
    t, tn, s, sn, q = make_points(8000, 40 + neq, "clustered")
    p, lmax = 6, 3
    ref_sem = semantics == 0
    pl = plan_for(ob, neq, p, lmax, t, tn, s, sn, semantics=semantics)
    v, g = pl.evaluate(q, f64=True)
    vo, go = oracle.oracle_fmm(t, s, q, neq=neq, p=p, lmax=lmax, tn=tn, sn=sn, ref_semantics=ref_sem,
                               eps2=oracle.EPS_REF if ref_sem else 0.0, exclude_self=not ref_sem)
    Mo, Lo = oracle.oracle_expansions(0), oracle.oracle_expansions(1)
    Mg, Lg = pl.expansions(0), pl.expansions(1)
    assert rel(Mg, Mo) < 1e-10
    assert rel(Lg, Lo) < 1e-10
    # the oracle accumulates outputs in float in reference semantics
    tol = 1e-6 if ref_sem else 1e-10
    assert rel(v, vo) < tol
    if neq == 0:
        assert rel(g.reshape(3, -1), go) < tol
    pl.close()


def test_direct_matches_oracle(ob, oracle):
    t, tn, s, sn, q = make_points(3000, 50)
    for neq in (0, 1, 2):
        pl = plan_for(ob, neq, 4, 2, t, tn, s, sn, semantics=1, exclude_self=True)
        v, g = pl.direct(q, 100, 600)
        vo, go = oracle.direct(t, s, q, neq=neq, eps2=0.0, exclude_self=True, tn=tn, sn=sn, targets=(100, 600))
        assert rel(v, vo) < 1e-12
        if neq == 0:
            assert rel(g, go) < 1e-12
        pl.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_accuracy_vs_fp64_direct(precision, ob, oracle):
    """Accurate semantics, p=12: relative error of the potential below 1e-6
    against the FP64 direct sum (self pairs excluded, no softening)."""
    n = 20000
    rng = np.random.default_rng(60)
    x = rng.random((3, n), dtype=np.float32)
    q = rng.uniform(-1, 1, n).astype(np.float32)
    pl = ob.Plan(kernel=0, p=12, lmax=3, precision=precision, semantics=1, exclude_self=True)
    pl.set_geometry(x, x, bbox=(0, 0, 0, 1))
    v, g = pl.evaluate(q, f64=True)
    vd, gd = oracle.direct(x, x, q, neq=0, eps2=0.0, exclude_self=True, targets=(0, 1024))
    assert rel(v[:1024], vd) < 1e-6
    assert rel(g.reshape(3, -1)[:, :1024], gd) < 1e-5
    pl.close()


def test_mixed_matches_fp64(ob):
    t, tn, s, sn, q = make_points(30000, 70, "clustered")
    for neq in (0, 1, 2):
        out = []
        for prec in (0, 1):
            pl = plan_for(ob, neq, 10, 4, t, tn, s, sn, semantics=1, precision=prec, exclude_self=True)
            out.append(pl.evaluate(q, f64=True))
            pl.close()
        assert rel(out[1][0], out[0][0]) < 1e-6


@pytest.mark.parametrize("lmax", [2, 3])
def test_mixed_near_field_large_leaves(lmax, ob):
    """Leaves of hundreds of points: several rounds of target groups per warp
    and source lists over many staged chunks (1e-6 vs FP64)."""
    t, tn, s, sn, q = make_points(40000, 71 + lmax)
    for neq in (0, 1, 2):
        out = []
        for prec in (0, 1):
            pl = plan_for(ob, neq, 8, lmax, t, tn, s, sn, semantics=1, precision=prec, exclude_self=True)
            out.append(pl.evaluate(q, f64=True))
            pl.close()
        assert rel(out[1][0], out[0][0]) < 1e-6
        if neq == 0:
            assert rel(out[1][1], out[0][1]) < 1e-6


def test_serial_phases_give_the_same_results(ob):
    t, tn, s, sn, q = make_points(20000, 75, "clustered")
    for prec in (0, 1):
        pl = plan_for(ob, 2, 10, 4, t, tn, s, sn, semantics=1, precision=prec, exclude_self=True)
        a = pl.evaluate(q, f64=True)[0]
        pl.set_overlap(False)
        b = pl.evaluate(q, f64=True)[0]
        ph = pl.timings()
        pl.set_overlap(True)
        c = pl.evaluate(q, f64=True)[0]
        pl.close()
        # the same sums (FP64 atomics in some translations: rounding order only;
        # in the mixed form an ulp of a multipole can move a rounding of its
        # FP16 split for the M2L, ~1e-10 at most)
        tol = 1e-13 if prec == 0 else 1e-9
        assert rel(b, a) < tol and rel(c, a) < tol
        assert ph["p2p"] > 0 and ph["m2l"] > 0


def test_host_and_device_pointers_agree(ob):
    torch = pytest.importorskip("torch")
    t, tn, s, sn, q = make_points(5000, 80)
    pl = plan_for(ob, 0, 8, 3, t, tn, s, sn)
    vh, gh = pl.evaluate(q)
    qd = torch.from_numpy(q).cuda()
    vd = torch.zeros(5000, device="cuda")
    gd = torch.zeros(15000, device="cuda")
    pl.evaluate(qd, vd, gd)
    torch.cuda.synchronize()
    # the M2L adds slot groups with FP64 atomics: equal to rounding
    assert rel(vd.cpu().numpy(), vh) < 1e-6
    assert rel(gd.cpu().numpy(), gh) < 1e-6
    # geometry from device tensors gives the same tree
    pl2 = ob.Plan(kernel=0, p=8, lmax=3)
    pl2.set_geometry(torch.from_numpy(t).cuda(), torch.from_numpy(s).cuda(), bbox=(0, 0, 0, 1))
    assert np.array_equal(pl2.tree(8), pl.tree(8))
    pl.close()
    pl2.close()


def test_errors_are_reported_not_fatal(ob):
    with pytest.raises(ob.FMMError):
        ob.Plan(p=0)
    with pytest.raises(ob.FMMError):
        ob.Plan(lmax=1)
    pl = ob.Plan(kernel=1)
    t, tn, s, sn, q = make_points(100, 90)
    with pytest.raises(ob.FMMError):  # Gni without target normals
        pl.set_geometry(t, s)
    with pytest.raises(ob.FMMError):  # evaluate before geometry
        pl.evaluate(q)
    pl.close()


@pytest.mark.parametrize("semantics,p", [(0, 10), (1, 10), (1, 12), (1, 15)])
def test_tensor_core_translations_match_fp64(semantics, p, ob):
    """The mixed form (FP32 P2M, tensor-core TF32x3 M2L, FP64 M2M/L2L) gives the
    FP64 multipoles and locals of every level to ~1e-6 (TF32x3 products carry
    ~2^-21 relative error, accumulated in FP32 over one pair's coefficients and
    in FP64 over pairs).  p = 12 and 15 (K = 169, 256) take the tensor-core path
    with two blocks of 128 output rows per operator; the FP32 sum over a pair's
    K = (p+1)^2 coefficients grows the locals' error like sqrt(K)."""
    t, tn, s, sn, q = make_points(40000, 100, "clustered")
    out = []
    for prec in (0, 1):
        pl = plan_for(ob, 0, p, 4, t, tn, s, sn, semantics=semantics, precision=prec)
        pl.evaluate(q, f64=True)
        out.append((pl.expansions(0), pl.expansions(1)))
        pl.close()
    assert rel(out[1][0], out[0][0]) < 1e-6
    assert rel(out[1][1], out[0][1]) < 2e-6 * max(1.0, ((p + 1) ** 2 / 121) ** 0.5)


def test_autotune_lmax_picks_a_measured_depth(ob):
    """fmmb_autotune_lmax times every depth of the range on the given geometry
    and returns the fastest one."""
    rng = np.random.default_rng(90)
    x = rng.random((3, 30000), dtype=np.float32)
    best, ms = ob.autotune_lmax(x, x, kernel=0, p=6, precision=1, semantics=1, exclude_self=True,
                                bbox=(0, 0, 0, 1), lmin=2, lmax=4, reps=2)
    assert set(ms) == {2, 3, 4} and all(v > 0 for v in ms.values())
    assert best == min(ms, key=ms.get)


@pytest.mark.parametrize("precision", [0, 1])
def test_laplace_g_without_gradient(precision, ob):
    """An evaluate of the G kernel with no gradient output (a NULL grad
    through the C ABI) gives the potential of the evaluate with gradient."""
    import ctypes
    t, tn, s, sn, q = make_points(20000, 92, "clustered")
    pl = plan_for(ob, 0, 10, 4, t, tn, s, sn, semantics=1, precision=precision, exclude_self=True)
    v, g = pl.evaluate(q, f64=True)
    pot = np.zeros(t.shape[1])
    for _ in range(2):  # the first call captures the no-gradient graph, the second replays it
        rc = ob.load().fmmb_evaluate_f64(pl._h, q.ctypes.data, pot.ctypes.data, None)
        assert rc == 0, ob.load().fmmb_last_error()
        # the same sums (FP64 atomics in the M2M: rounding order only; in the
        # mixed form an ulp of a multipole can move a rounding of its FP16 split)
        assert rel(pot, v) < (1e-13 if precision == 0 else 1e-9)
    pl.close()


def test_autotune_order_meets_the_tolerance(ob):
    """fmmb_autotune_order: the lowest order in the range whose FMM meets the
    tolerance against the FP64 direct sum on its sample of targets, at the
    depth fmmb_autotune_lmax picks for it; the order below misses it, and the
    chosen plan meets it on targets outside the sample too."""
    t, _, _, _, q = make_points(30000, 91, "clustered")
    kw = dict(kernel=0, precision=ob.MIXED, semantics=ob.SEM_ACCURATE, exclude_self=True, bbox=(0, 0, 0, 1))
    p, lmax, err, ms = ob.autotune_order(t, t, 1e-6, p_lo=6, p_hi=14, **kw)
    assert 6 < p <= 14 and err <= 1e-6 and 2 <= lmax <= 10 and ms > 0
    _, _, err_below, _ = ob.autotune_order(t, t, 1e-6, p_lo=p - 1, p_hi=p - 1, **kw)
    assert err_below > 1e-6
    pl = ob.Plan(kernel=0, p=p, lmax=lmax, precision=ob.MIXED, semantics=ob.SEM_ACCURATE, exclude_self=True)
    pl.set_geometry(t, t, bbox=(0, 0, 0, 1))
    v, _ = pl.evaluate(q, f64=True)
    vd, _ = pl.direct(q, 20000, 21000)
    pl.close()
    assert rel(v[20000:21000], vd) < 2e-6
    # a tolerance no order in the range reaches: the last order, its error reported
    p2, _, err2, _ = ob.autotune_order(t, t, 1e-14, p_lo=4, p_hi=5, **kw)
    assert p2 == 5 and err2 > 1e-14
    with pytest.raises(ob.FMMError):
        ob.autotune_order(t, t, 1e-6, p_lo=8, p_hi=4, **kw)


@pytest.mark.parametrize("precision", [0, 1])
def test_many_right_hand_sides_equal_single_evaluates(precision, ob):
    """nrhs = 3 in one evaluate gives the three single evaluates, gradients
    included: FP64 form (each right-hand side replayed through the plan's CUDA
    graph) to 1e-12; mixed form (the near field of all three in one pass,
    p2p_multi.cu, summing FP32 terms over 128 sources instead of 32 before
    the FP64 accumulation; the far field per right-hand side) to 1e-6."""
    t, tn, s, sn, q = make_points(12000, 110, "clustered")
    rng = np.random.default_rng(111)
    qs = rng.uniform(-1, 1, (3, s.shape[1])).astype(np.float32)
    kw = dict(semantics=1, precision=precision, exclude_self=True)
    pl = plan_for(ob, 0, 8, 4, t, tn, s, sn, nrhs=3, **kw)
    v3, g3 = pl.evaluate(qs.ravel(), f64=True)
    pl.close()
    one = plan_for(ob, 0, 8, 4, t, tn, s, sn, **kw)
    tol = 1e-12 if precision == 0 else 1e-6
    for r in range(3):
        v, g = one.evaluate(qs[r], f64=True)
        assert rel(v3[r * 12000:(r + 1) * 12000], v) < tol
        assert rel(g3.reshape(3, 3, -1)[r], g.reshape(3, -1)) < tol
    one.close()


@pytest.mark.parametrize("neq", [0, 1, 2])
def test_many_rhs_near_field_vs_direct(neq, ob, oracle):
    """The all-right-hand-side near field (nrhs = 9: groups of 8 and 1) within
    the FMM's accuracy of the FP64 direct sum for every right-hand side."""
    t, tn, s, sn, q = make_points(8000, 120 + neq, "clustered")
    rng = np.random.default_rng(121)
    qs = rng.uniform(-1, 1, (9, 8000)).astype(np.float32)
    pl = plan_for(ob, neq, 12, 3, t, tn, s, sn, nrhs=9, semantics=1, precision=1, exclude_self=True)
    v, _ = pl.evaluate(qs.ravel(), f64=True)
    pl.close()
    for r in (0, 7, 8):
        ref, _ = oracle.direct(t, s, qs[r], neq=neq, eps2=0.0, exclude_self=True, tn=tn, sn=sn, targets=(0, 1000))
        assert rel(v[r * 8000:r * 8000 + 1000], ref) < 5e-6


def _bench_sphere():
    from old_fmm_bem_b200 import geometry
    x, n, q = geometry.bem_double_layer_problem(6, seed=0)
    return x, q


def _bench_clusters(n):
    rng = np.random.default_rng(13)
    c = rng.uniform(0.1, 0.9, (3, 32))
    lab = rng.integers(0, 32, 1 << 20)
    x = np.clip(c[:, lab] + 0.02 * rng.standard_normal((3, 1 << 20)), 0.0, 1.0).astype(np.float32)
    q = rng.standard_normal(1 << 20).astype(np.float32)
    return np.ascontiguousarray(x[:, :n]), q[:n].copy()


@pytest.mark.parametrize("case", ["sphere245760_lmax5", "clustered262144_lmax6"])
def test_tree_bit_exact_vs_reference_at_benchmark_sizes(case, ob, oracle):
    """Permutations, leaf ranges and every interaction list bit-exact against
    the reference library itself (its boxn / csort / boxdata / boxm2m / ijbox
    compiled from source, oracle/_ref) on the geometries the benchmarks run:
    the 245,760-point icosphere at depth 5 (uneven leaves, most boxes empty)
    and 262,144 points of the 32-cluster distribution at depth 6; potentials of
    the FP64 form (reference semantics, p = 8) against the reference's float
    outputs to 1e-6."""
    if not oracle.ref_available(8):
        pytest.skip("reference library not built (oracle/_ref)")
    if case.startswith("sphere"):
        x, q = _bench_sphere()
        lmax = 5
        lo = x.min(axis=1)
        bb = (float(lo[0]), float(lo[1]), float(lo[2]), float((x.max(axis=1) - lo).max() * (1 + 1e-5)))
    else:
        x, q = _bench_clusters(262144)
        lmax = 6
        bb = (0.0, 0.0, 0.0, 1.0)
    vr, gr = oracle.ref_fmm(x, x, q, neq=0, p=8, lmax=lmax, bbox=bb)
    rr = oracle.ref_records(8)
    pl = plan_for(ob, 0, 8, lmax, x, None, x, None, bbox=bb)
    for k in (0, 1, 6, 7):
        assert np.array_equal(pl.tree(k), rr[k]), k
    la, lb = oracle.parse_lists(pl.tree(8)), oracle.parse_lists(rr[8])
    assert len(la) == len(lb)
    for a, b in zip(la, lb):
        assert a[0] == b[0] and a[1] == b[1] and a[3] == b[3]
    v, g = pl.evaluate(q, f64=True)
    assert rel(v, vr.astype(np.float64)) < 1e-6
    assert rel(g.reshape(3, -1), gr.astype(np.float64)) < 1e-6
    pl.close()
