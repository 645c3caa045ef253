"""The BEM solvation driver (old_fmm_bem_b200/bem.py, the reference's
bio/main.cxx pipeline): MSMS readers, panel geometry, and the physics of the
formulation, on the CPU with the dense checker of oracle/bem_oracle.py.

* readers: a mesh written by write_msms reads back exactly; the reference's
  own fixtures (bio/data/sphere.*, tripeptide.*, read in place when the
  reference tree is present) parse to their line counts, and the reference's
  panel orientation, (p2 - p0) x (p1 - p0), is opposite to the MSMS vertex
  normals on every panel (the formulation's convention);
* physics: a unit charge at the centre of a sphere of radius 5 (e1 = 4,
  e2 = 20) gives the Born energy -0.5 * 332.112 / 5 * (1/4 - 1/20) within the
  discretisation error of one centroid per panel (3 % at 1,280 panels).
"""
import os

import numpy as np
import pytest

from conftest import reference_root
from old_fmm_bem_b200 import bem, geometry

REF_DATA = os.path.join(reference_root(), "bio", "data")


def test_msms_round_trip(tmp_path):
    v, f = geometry.geodesic_sphere(4, radius=5.0)
    xa = np.array([[0.5, -1.0], [0.2, 0.3], [0.0, 1.1]], np.float32)
    qa = np.array([1.0, -0.5], np.float32)
    stem = str(tmp_path / "mesh")
    bem.write_msms(stem, v, f, xa, qa)
    v2, f2 = bem.read_vert(stem + ".vert"), bem.read_face(stem + ".face")
    xa2, qa2 = bem.read_xyzq(stem + ".xyzq")
    assert np.array_equal(f2, f) and np.allclose(v2, v, atol=1e-5)
    assert np.allclose(xa2, xa) and np.allclose(qa2, qa)


@pytest.mark.skipif(not os.path.isdir(REF_DATA), reason="reference fixtures not present")
@pytest.mark.parametrize("name,nv,nf,nq", [("sphere", 290, 576, 20), ("tripeptide", 1986, 3968, 44)])
def test_reference_fixtures_parse(name, nv, nf, nq):
    v = bem.read_vert(os.path.join(REF_DATA, name + ".vert"))
    f = bem.read_face(os.path.join(REF_DATA, name + ".face"))
    xa, qa = bem.read_xyzq(os.path.join(REF_DATA, name + ".xyzq"))
    assert v.shape == (nv, 3) and f.shape == (nf, 3) and xa.shape == (3, nq) and qa.shape == (nq,)
    assert f.min() == 0 and f.max() == nv - 1
    cen, nrm, area = bem.panels(v, f)
    assert np.all(area > 1e-5) and np.allclose(np.linalg.norm(nrm, axis=0), 1.0, atol=1e-5)
    vn = np.loadtxt(os.path.join(REF_DATA, name + ".vert"), usecols=(3, 4, 5))
    p0, p1, p2 = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    keep = 0.5 * np.linalg.norm(np.cross(p2 - p0, p1 - p0), axis=1) > 1e-5
    assert np.all(np.einsum("ij,ji->j", vn[f[keep]].mean(axis=1), nrm) < 0)


def test_dense_pipeline_gives_born_energy():
    from oracle import bem_oracle
    v, f = geometry.geodesic_sphere(8, radius=5.0)
    cen, nrm, area = bem.panels(v, f)
    E, _, _ = bem_oracle.solvation_energy_dense(cen, nrm, area, np.zeros((3, 1), np.float32), np.ones(1, np.float32))
    born = -0.5 * bem.COULOMB / 5.0 * (1 / geometry.E1 - 1 / geometry.E2)
    assert abs(E - born) < 0.03 * abs(born)
