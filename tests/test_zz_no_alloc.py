"""fmmb_direct_static (the entry point that allocates nothing) against the plan's
fmmb_direct_f64 on the same inputs, through the C ABI.

Both sum in FP64; fmmb_direct_static adds its source-split partials in a
different order and rounds to float, so each output must lie within one float
ulp of fmmb_direct_f64's FP64 value rounded to float (plus 1e-12 of the
largest output, for the reordering noise of outputs near zero).  Two calls in a row (the
second smaller in ni, with more source splits) check that nothing of the first
call's scratch contents leaks into the second; a repeat of the first call must
reproduce it bit for bit.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def ob():
    import old_fmm_bem_b200 as ob
    from old_fmm_bem_b200 import build
    build.build()
    ob.load()
    return ob


def _points(seed, ni, nj, dup):
    rng = np.random.default_rng(seed)
    t = rng.random((3, ni), dtype=np.float32)
    s = rng.random((3, nj), dtype=np.float32)
    s[:, :dup] = t[:, :dup]  # coincident pairs exercise exclude_self / eps
    tn = rng.standard_normal((3, ni)).astype(np.float32)
    sn = rng.standard_normal((3, nj)).astype(np.float32)
    q = rng.uniform(-1, 1, nj).astype(np.float32)
    return t, tn, s, sn, q


def _cfg(ob, kernel, semantics, exclude_self):
    cfg = ob._Config()
    ob.load().fmmb_config_init(ctypes.byref(cfg))
    cfg.kernel, cfg.semantics, cfg.exclude_self, cfg.eps2 = kernel, semantics, exclude_self, 0.0
    return cfg


def _static(ob, kernel, semantics, exclude_self, t, tn, s, sn, q):
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    T, TN, S, SN, Q = dev(t), dev(tn), dev(s), dev(sn), dev(q)
    ni, nj = t.shape[1], s.shape[1]
    pot = torch.full((ni,), float("nan"), device="cuda")
    grad = torch.full((3 * ni,), float("nan"), device="cuda") if kernel == 0 else None
    cfg = _cfg(ob, kernel, semantics, exclude_self)
    rc = ob.load().fmmb_direct_static(ctypes.byref(cfg), ni, T[0].data_ptr(), T[1].data_ptr(), T[2].data_ptr(),
                                      TN[0].data_ptr(), TN[1].data_ptr(), TN[2].data_ptr(), nj, S[0].data_ptr(),
                                      S[1].data_ptr(), S[2].data_ptr(), SN[0].data_ptr(), SN[1].data_ptr(),
                                      SN[2].data_ptr(), Q.data_ptr(), pot.data_ptr(),
                                      grad.data_ptr() if grad is not None else None,
                                      torch.cuda.current_stream().cuda_stream or 1)
    assert rc == 0, ob.load().fmmb_last_error()
    torch.cuda.synchronize()
    return pot.cpu().numpy(), (grad.cpu().numpy().reshape(3, ni) if grad is not None else None)


def _plan_direct(ob, kernel, semantics, exclude_self, t, tn, s, sn, q):
    pl = ob.Plan(kernel=kernel, p=4, lmax=2, semantics=semantics, exclude_self=bool(exclude_self))
    pl.set_geometry(t, s, tn if kernel == 1 else None, sn if kernel == 2 else None)
    v, g = pl.direct(q)
    pl.close()
    return v, g


def _within_one_ulp(a, ref64):
    ref32 = ref64.astype(np.float32)
    assert np.all(np.isfinite(a))
    # one ulp, plus FP64 reordering noise for the few outputs near zero
    tol = np.spacing(np.abs(ref32)).astype(np.float64) + 1e-12 * np.abs(ref64).max()
    assert np.all(np.abs(a.astype(np.float64) - ref32.astype(np.float64)) <= tol)


CASES = [
    # kernel, semantics, exclude_self, seed, ni, nj, coincident pairs
    (0, 1, 1, 1, 20000, 9000, 500),
    (2, 0, 0, 2, 3000, 40000, 300),
]


def test_two_calls_in_a_row_match_direct_f64(ob):
    first = None
    for kernel, sem, excl, seed, ni, nj, dup in CASES:
        t, tn, s, sn, q = _points(seed, ni, nj, dup)
        v, g = _static(ob, kernel, sem, excl, t, tn, s, sn, q)
        vr, gr = _plan_direct(ob, kernel, sem, excl, t, tn, s, sn, q)
        _within_one_ulp(v, vr)
        if kernel == 0:
            _within_one_ulp(g, gr)
        if first is None:
            first = (v, g)
    # the first case again, after the second call left its partials behind
    kernel, sem, excl, seed, ni, nj, dup = CASES[0]
    v, g = _static(ob, kernel, sem, excl, *_points(seed, ni, nj, dup))
    assert np.array_equal(v, first[0]) and np.array_equal(g, first[1])


def test_gni_and_oversize_rejected(ob):
    t, tn, s, sn, q = _points(3, 5000, 6000, 0)
    v, _ = _static(ob, 1, 1, 1, t, tn, s, sn, q)
    vr, _ = _plan_direct(ob, 1, 1, 1, t, tn, s, sn, q)
    _within_one_ulp(v, vr)
    # 4 x ni partial sums beyond FMMB_STATIC_SCRATCH_BYTES / 8: rejected before any GPU work
    lib = ob.load()
    cap = (16 << 20) // 8
    ni = cap // 4 + 1
    buf = torch.zeros(8, device="cuda")
    p = buf.data_ptr()
    cfg = _cfg(ob, 0, 1, 1)
    rc = lib.fmmb_direct_static(ctypes.byref(cfg), ni, p, p, p, None, None, None, 8, p, p, p, None, None, None, p,
                                p, p, None)
    assert rc == -4 and b"static scratch" in lib.fmmb_last_error()
    # host pointers are refused (no staging copies, which would allocate)
    h = np.zeros(8, np.float32)
    hp = h.ctypes.data
    rc = lib.fmmb_direct_static(ctypes.byref(cfg), 8, hp, hp, hp, None, None, None, 8, hp, hp, hp, None, None, None,
                                hp, hp, None, None)
    assert rc == -1 and b"device" in lib.fmmb_last_error()


@pytest.mark.skipif(not torch.cuda.is_available() or torch.cuda.device_count() < 2, reason="needs two GPUs")
def test_other_device_memory_rejected(ob):
    """Memory of another GPU is refused before any GPU work: the kernels would
    run on the current device and read it as a peer access nobody enabled."""
    lib = ob.load()
    cfg = _cfg(ob, 0, 1, 1)
    other = torch.zeros(8, device="cuda:1")
    op = other.data_ptr()
    with torch.cuda.device(0):
        rc = lib.fmmb_direct_static(ctypes.byref(cfg), 8, op, op, op, None, None, None, 8, op, op, op, None, None,
                                    None, op, op, None, None)
    assert rc == -1 and b"current device" in lib.fmmb_last_error()
