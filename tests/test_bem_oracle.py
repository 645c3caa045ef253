"""The BEM checker (oracle/bem_oracle.py) and the batch geometry, on the CPU.

* the dense kernel matrices reproduce the oracle's C direct sum (pinned to the
  reference's golden vectors) to 1e-12;
* the numpy GMRES converges to numpy.linalg.solve on a small BEM system, and
  its fixed-iteration iterates reduce the residual monotonically;
* geodesic spheres have 20 freq^2 outward triangles whose areas approach 4 pi.
"""
import numpy as np
import pytest

from old_fmm_bem_b200 import geometry


def _sphere(freq):
    v, f = geometry.geodesic_sphere(freq)
    x, n, w, _ = geometry.quadrature_points(v, f, "centroid")
    return x, n, w


@pytest.mark.parametrize("kernel", [0, 1, 2])
def test_kernel_matrix_matches_c_direct(kernel, oracle):
    from oracle import bem_oracle
    x, n, w = _sphere(5)
    q = np.random.default_rng(kernel).uniform(-1, 1, x.shape[1]).astype(np.float32)
    K = bem_oracle.kernel_matrix(x, kernel, nt=n if kernel == 1 else None, ns=n if kernel == 2 else None)
    ref, _ = oracle.direct(x, x, q, neq=kernel, eps2=0.0, exclude_self=True, tn=n if kernel == 1 else None,
                           sn=n if kernel == 2 else None)
    got = K @ q.astype(np.float64)
    assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref)


@pytest.mark.parametrize("kernel", [1, 2])
def test_gmres_oracle_converges_to_dense_solve(kernel):
    from oracle import bem_oracle
    x, n, area = _sphere(6)
    A = bem_oracle.bem_matrix(x, n, area / geometry.E1, kernel, geometry.BEM_DIAG)
    b = np.random.default_rng(3).uniform(-1, 1, len(area))
    xs = np.linalg.solve(A, b)
    xg, it, rel = bem_oracle.gmres(A, b, precond=1 / geometry.BEM_DIAG, restart=12, max_iter=300, rtol=1e-13)
    assert rel <= 1e-13 and it < 300
    assert np.linalg.norm(xg - xs) <= 1e-10 * np.linalg.norm(xs)
    # fixed iteration counts: the preconditioned residual does not grow
    last = np.inf
    for k in (2, 5, 10, 20):
        xk, itk, relk = bem_oracle.gmres(A, b, precond=1 / geometry.BEM_DIAG, restart=30, max_iter=k)
        r = np.linalg.norm(b - A @ xk)
        assert itk == k and r <= last * (1 + 1e-12) + 1e-12 * np.linalg.norm(b)
        last = r


def test_geodesic_sphere():
    for freq in (1, 3, 7):
        v, f = geometry.geodesic_sphere(freq)
        assert f.shape == (20 * freq * freq, 3)
        assert np.allclose(np.linalg.norm(v, axis=1), 1.0)
        x, n, w, _ = geometry.quadrature_points(v, f, "centroid")
        assert np.all(np.einsum("ij,ij->j", x.astype(np.float64), n.astype(np.float64)) > 0)  # outward
    x, n, w = _sphere(40)
    assert abs(w.sum() - 4 * np.pi) < 2e-3 * 4 * np.pi
    probs = geometry.bem_batch_problems(8, seed=1)
    assert len(probs) == 8 and all(2000 * 0.8 <= p[0].shape[1] <= 200000 * 1.2 for p in probs)
