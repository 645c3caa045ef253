"""The 6-node boundary-element geometry of the reference's biobem solver
(old_fmm_bem_b200/mesh6.py) against the reference itself: its
biobem/geometry.cxx and biobem/bem3d.cxx compiled from source, run on the
reference's sphere mesh (tests/golden/ref_mesh6_sphere.npz, made by
tests/golden/make_mesh6_golden.py).

* rules of 1, 3, 4 and 6 points: every array bit-identical to the
  reference's -- node coordinates and numbering, the elements around each
  node, the rule, element areas, metric x weight, shape functions, node
  normals and tangents;
* rules of 7, 9, 12 and 13 points (where the reference's elm_geom writes past
  its 6-entry work arrays and its outputs are undefined): the same areas as the
  6-point rule to 1e-6, unit normals, shape functions summing to 1, and each
  rule integrating the monomials of its degree exactly on the triangle.
"""
import os

import numpy as np
import pytest

from old_fmm_bem_b200 import mesh6

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_mesh6_sphere.npz")


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(GOLD))


@pytest.fixture(scope="module")
def mesh(gold):
    return mesh6.six_node_mesh(gold["vert"], gold["face"], gold["xyzq"])


def test_mesh_matches_reference(gold, mesh):
    assert np.array_equal(mesh["ptr"], gold["ptr"])
    assert np.array_equal(mesh["ntr"], gold["ntr"])
    assert np.array_equal(mesh["xq"], gold["xq"]) and np.array_equal(mesh["vq"], gold["vq"])
    cnt = np.diff(mesh["nne_ptr"])
    assert np.array_equal(cnt, gold["nne"][:, 0])
    for i in range(len(cnt)):  # the first 8 element numbers the reference keeps in its 9-column record
        k = min(int(cnt[i]), 8)
        assert np.array_equal(mesh["nne_elm"][mesh["nne_ptr"][i]:mesh["nne_ptr"][i] + k], gold["nne"][i, 1:1 + k])


@pytest.mark.parametrize("ngl", [1, 3, 4, 6])
def test_element_geometry_bit_exact(ngl, gold, mesh):
    g = mesh6.element_geometry(mesh, ngl)
    for k in ("xiq", "etq", "wq", "are", "hsg"):
        assert np.array_equal(g[k], gold[f"{k}_{ngl}"]), k
    assert np.array_equal(g["phi"], gold[f"phi_{ngl}"])
    for k in ("vna", "vta", "vsa"):
        assert np.array_equal(g[k], gold[k]), k


@pytest.mark.parametrize("ngl", [7, 9, 12, 13])
def test_higher_rules_consistent(ngl, mesh):
    g6 = mesh6.element_geometry(mesh, 6)
    g = mesh6.element_geometry(mesh, ngl)
    a6, a = g6["are"].astype(np.float64), g["are"].astype(np.float64)
    assert np.abs(a - a6).max() / a6.max() < 1e-6
    assert np.allclose(np.linalg.norm(g["vna"].astype(np.float64), axis=1), 1.0, atol=1e-6)
    assert np.array_equal(g["vna"], g6["vna"])  # node normals do not depend on the rule
    assert np.allclose(g["phi"].astype(np.float64).sum(-1), 1.0, atol=1e-6)


@pytest.mark.parametrize("ngl,degree", [(1, 1), (3, 2), (4, 3), (6, 4), (7, 5), (9, 5), (12, 6), (13, 7)])
def test_rules_integrate_their_degree(ngl, degree):
    """sum_j w_j xi^a eta^b = 2 * a! b! / (a + b + 2)!, the mean of xi^a eta^b
    over the reference triangle (weights sum to 1)."""
    from math import factorial
    xi, eta, w = (v.astype(np.float64) for v in mesh6.triangle_rule(ngl))
    for a in range(degree + 1):
        for b in range(degree + 1 - a):
            exact = 2.0 * factorial(a) * factorial(b) / factorial(a + b + 2)
            assert abs(np.sum(w * xi ** a * eta ** b) - exact) < 2e-7, (a, b)
