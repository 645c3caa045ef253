"""Generate tests/golden/ref_mesh6_sphere.npz: the reference's own 6-node
boundary-element geometry (biobem/geometry.cxx, biobem/bem3d.cxx, compiled from
its sources by oracle/Makefile into oracle/_ref/bem3d_ref_ngl<n>) on the
reference's sphere mesh (bio/data/sphere.vert / .face / .xyzq), with that
mesh as the fixture's input.  Run in a container that has the reference
sources:

    make -f oracle/Makefile bem3d && python tests/golden/make_mesh6_golden.py

Only the rules of 1, 3, 4 and 6 points are recorded: with more points the
reference's elm_geom writes past its 6-entry work arrays (biobem/bem3d.cxx:331-332,
indexed by the quadrature point) and its results are undefined.
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
from conftest import reference_root  # noqa: E402

NGLS = (1, 3, 4, 6)


def read_output(path):
    """The binary written by oracle/refshim/src/bem3d_driver.cpp."""
    b = open(path, "rb").read()
    off = 0

    def take(dt, n):
        nonlocal off
        a = np.frombuffer(b, dt, n, off)
        off += a.nbytes
        return a.copy()

    nwe, nwn, nch, ngl = (int(v) for v in take(np.int32, 4))
    r = {"ptr": take(np.float32, nwn * 3).reshape(nwn, 3), "ntr": take(np.int32, nwe * 6).reshape(nwe, 6),
         "nne": take(np.int32, nwn * 9).reshape(nwn, 9)}
    for k in ("xiq", "etq", "wq"):
        r[k] = take(np.float32, ngl)
    r["are"] = take(np.float32, nwe)
    tabs = [take(np.float32, nwe * ngl).reshape(nwe, ngl) for _ in range(7)]
    r["hsg"], r["phi"] = tabs[0], np.stack(tabs[1:], -1)
    for k in ("vna", "vta", "vsa"):
        r[k] = take(np.float32, nwn * 3).reshape(nwn, 3)
    q = [take(np.float32, nch) for _ in range(4)]
    r["xq"], r["vq"] = np.stack(q[:3]), q[3]
    return r


def main():
    ref = reference_root()
    data = os.path.join(ref, "bio", "data", "sphere")
    out = {"vert": np.loadtxt(data + ".vert", usecols=(0, 1, 2)),
           "face": np.loadtxt(data + ".face", usecols=(0, 1, 2), dtype=np.int64),
           "xyzq": np.loadtxt(data + ".xyzq", usecols=(0, 1, 2, 3))}
    with tempfile.TemporaryDirectory() as tmp:
        for ngl in NGLS:
            path = os.path.join(tmp, "out.bin")
            subprocess.run([os.path.join(ROOT, "oracle", "_ref", f"bem3d_ref_ngl{ngl}"), path],
                           cwd=os.path.join(ref, "biobem"), check=True)
            r = read_output(path)
            for k, v in r.items():
                if k in ("ptr", "ntr", "nne", "vna", "vta", "vsa", "xq", "vq") and ngl != NGLS[0]:
                    assert np.array_equal(out[k], v), k  # independent of the rule
                    continue
                out[k if k in ("ptr", "ntr", "nne", "vna", "vta", "vsa", "xq", "vq") else f"{k}_{ngl}"] = v
    np.savez_compressed(os.path.join(HERE, "ref_mesh6_sphere.npz"), **out)


if __name__ == "__main__":
    main()
