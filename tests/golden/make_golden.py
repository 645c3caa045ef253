"""Generate tests/golden/ref_fmm_*.npz: seeded inputs and the outputs of the
reference's own CPU fmm() (compiled from its sources by oracle/Makefile into
oracle/_ref).  Run in a container that has the reference sources:

    make -f oracle/Makefile all && python tests/golden/make_golden.py

The fixtures pin the oracle restatement where the reference library is not
available (tests/test_oracle_pin.py).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import pyoracle as po  # noqa: E402

CASES = [  # (name, N, lmax, p, seed)
    ("n2000_l2_p8", 2000, 2, 8, 11),
    ("n6000_l3_p8", 6000, 3, 8, 12),
    ("n6000_l3_p10", 6000, 3, 10, 13),
]


def inputs(n, seed):
    rng = np.random.default_rng(seed)
    t = rng.random((3, n), dtype=np.float32)
    s = rng.random((3, n), dtype=np.float32)
    tn = rng.standard_normal((3, n)).astype(np.float32)
    tn /= np.linalg.norm(tn, axis=0)
    sn = rng.standard_normal((3, n)).astype(np.float32)
    sn /= np.linalg.norm(sn, axis=0)
    q = rng.uniform(-1, 1, n).astype(np.float32)
    return t, tn, s, sn, q


def main():
    for name, n, lmax, p, seed in CASES:
        t, tn, s, sn, q = inputs(n, seed)
        out = dict(t=t, tn=tn, s=s, sn=sn, q=q, lmax=lmax, p=p)
        for neq in (0, 1, 2):
            v, g = po.ref_fmm(t, s, q, neq=neq, p=p, lmax=lmax, tn=tn, sn=sn)
            out[f"v{neq}"] = v
            if g is not None:
                out[f"g{neq}"] = g
            rec = po.ref_records(p)
            if neq == 0:
                out["perm_i"], out["perm_j"] = rec[0], rec[1]
                out["leaf_i"], out["leaf_j"] = rec[6], rec[7]
                out["lists"] = rec[8]
        path = os.path.join(HERE, f"ref_fmm_{name}.npz")
        np.savez_compressed(path, **out)
        print("wrote", path, os.path.getsize(path))


if __name__ == "__main__":
    main()
