"""Pin the oracle restatement (oracle/fmm_oracle.cpp) to the reference.

Two sources of truth:
* the committed golden fixtures tests/golden/ref_fmm_*.npz, made by
  tests/golden/make_golden.py from the reference's own fmm() compiled from its
  sources (always available);
* the reference library oracle/_ref/libfmmref_mp*.so itself, on fresh seeded
  inputs (where it has been built).

Trees, permutations and interaction lists must be identical; potentials and
gradients agree to the float rounding of the reference's outputs.
"""
import glob
import os

import numpy as np
import pytest

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "ref_fmm_*.npz")))


def _lists_equal(a, b, po):
    la, lb = po.parse_lists(a), po.parse_lists(b)
    return len(la) == len(lb) and all(x[0] == y[0] and x[1] == y[1] and x[3] == y[3] for x, y in zip(la, lb))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_oracle_matches_golden(path, oracle):
    d = np.load(path)
    p, lmax = int(d["p"]), int(d["lmax"])
    for neq in (0, 1, 2):
        v, g = oracle.oracle_fmm(d["t"], d["s"], d["q"], neq=neq, p=p, lmax=lmax, tn=d["tn"], sn=d["sn"])
        ref = d[f"v{neq}"].astype(np.float64)
        assert np.max(np.abs(v - ref)) <= 2e-7 * np.max(np.abs(ref))
        # the large majority of outputs is bit-identical in float
        assert np.mean(v.astype(np.float32) == d[f"v{neq}"]) > 0.9
        if neq == 0:
            gr = d["g0"].astype(np.float64)
            assert np.max(np.abs(g - gr)) <= 2e-7 * np.max(np.abs(gr))
            rec = oracle.oracle_records()
            assert np.array_equal(rec[0], d["perm_i"]) and np.array_equal(rec[1], d["perm_j"])
            assert np.array_equal(rec[6], d["leaf_i"]) and np.array_equal(rec[7], d["leaf_j"])
            assert _lists_equal(rec[8], d["lists"], oracle)


@pytest.mark.parametrize("n,lmax,p", [(3000, 2, 8), (12000, 3, 10)])
def test_oracle_matches_reference_build(n, lmax, p, oracle):
    if not oracle.ref_available(p):
        pytest.skip("reference library not built (oracle/_ref)")
    rng = np.random.default_rng(100 + n)
    # clustered points: uneven leaves, empty boxes, boxes on the root boundary
    c = rng.random((3, 8))
    t = np.clip(c[:, rng.integers(0, 8, n)] + 0.08 * rng.standard_normal((3, n)), 0, 1).astype(np.float32)
    s = np.clip(c[:, rng.integers(0, 8, n)] + 0.08 * rng.standard_normal((3, n)), 0, 1).astype(np.float32)
    tn = rng.standard_normal((3, n)).astype(np.float32)
    sn = rng.standard_normal((3, n)).astype(np.float32)
    q = rng.uniform(-1, 1, n).astype(np.float32)
    for neq in (0, 1, 2):
        vr, gr = oracle.ref_fmm(t, s, q, neq=neq, p=p, lmax=lmax, tn=tn, sn=sn)
        rr = oracle.ref_records(p)
        vo, go = oracle.oracle_fmm(t, s, q, neq=neq, p=p, lmax=lmax, tn=tn, sn=sn)
        ro = oracle.oracle_records()
        for k in (0, 1, 6, 7):
            assert np.array_equal(rr[k], ro[k]), k
        assert _lists_equal(rr[8], ro[8], oracle)
        assert np.max(np.abs(vo - vr)) <= 2e-7 * np.max(np.abs(vr))
        if neq == 0:
            assert np.max(np.abs(go - gr)) <= 2e-7 * np.max(np.abs(gr))


def test_oracle_fmm_accuracy_vs_direct(oracle):
    """Accurate semantics (exact angles, no softening, self pairs skipped):
    the restated FMM converges to the FP64 direct sum as p grows."""
    rng = np.random.default_rng(7)
    n = 8000
    x = rng.random((3, n), dtype=np.float32)
    q = rng.uniform(-1, 1, n).astype(np.float32)
    ref, gref = oracle.direct(x, x, q, neq=0, eps2=0.0, exclude_self=True, targets=(0, 512))
    errs = []
    for p in (4, 8, 12):
        v, g = oracle.oracle_fmm(x, x, q, neq=0, p=p, lmax=3, ref_semantics=False, exclude_self=True)
        errs.append(np.linalg.norm(v[:512] - ref) / np.linalg.norm(ref))
    assert errs[0] > errs[1] > errs[2]
    assert errs[2] < 1e-6
