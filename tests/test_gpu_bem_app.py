"""The BEM solvation pipeline on the GPU (old_fmm_bem_b200/bem.py: two FMM
plans, a Gni plan and fmmb_gmres) against the same pipeline with dense FP64
matrices and a direct solve (oracle/bem_oracle.py), on MSMS files written and
read back.  Tolerances (GMRES rtol 1e-9): the energy to 1e-6 (FP64 form) /
1e-5 (mixed); the surface density to 1e-4 in both, the truncation error of
the normal-derivative kernel on the surface at p = 12 (a few 1e-5, which the
energy, a weighted integral of the density, averages out).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mesh(tmp_path):
    from old_fmm_bem_b200 import bem, geometry
    v, f = geometry.geodesic_sphere(14, radius=5.0)  # 3,920 panels
    rng = np.random.default_rng(3)
    xa = (rng.uniform(-1, 1, (3, 12)) * 2.5).astype(np.float32)
    qa = rng.choice([-1.0, 1.0], 12).astype(np.float32)
    stem = str(tmp_path / "mol")
    bem.write_msms(stem, v, f, xa, qa)
    return bem.read_vert(stem + ".vert"), bem.read_face(stem + ".face"), *bem.read_xyzq(stem + ".xyzq")


@pytest.mark.parametrize("precision", [0, 1])
def test_solvation_energy_matches_dense(precision, tmp_path):
    import old_fmm_bem_b200  # noqa: F401  (builds on import of bem)
    from old_fmm_bem_b200 import bem, build
    from oracle import bem_oracle
    build.build()
    v, f, xa, qa = _mesh(tmp_path)
    E, info = bem.solvation_energy(v, f, xa, qa, p=12, precision=precision, rtol=1e-9, max_iter=100)
    cen, nrm, area = bem.panels(v, f)
    Ed, xd, _ = bem_oracle.solvation_energy_dense(cen, nrm, area, xa, qa)
    tol_e, tol_x = (1e-6, 1e-4) if precision == 0 else (1e-5, 1e-4)
    # rel_resid is the residual of the returned density through the FMM itself:
    # at the iteration's own level in FP64, at the mixed matvec's rounding level
    # (relative ~1e-7 of A x) in the mixed form
    assert info["iterations"] < 100 and info["rel_resid"] <= (1e-9 if precision == 0 else 1e-5)
    assert abs(E - Ed) <= tol_e * abs(Ed)
    assert np.linalg.norm(info["density"] - xd) <= tol_x * np.linalg.norm(xd)
