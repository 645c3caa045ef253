"""The C-ABI library builds, loads and exports exactly what include/fmmb.h
declares (no GPU needed: nothing here runs a kernel)."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "fmmb.h")).read()
    return sorted(set(re.findall(r"FMMB_API\s+[\w\s\*]+?\b(fmmb_\w+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from old_fmm_bem_b200 import build
    path = build.build()
    return ctypes.CDLL(path), path


def test_header_declares_api():
    names = _declared()
    assert "fmmb_plan_create" in names and "fmmb_evaluate" in names and len(names) >= 15


def test_library_exports_every_declared_symbol(lib):
    handle, path = lib
    for name in _declared():
        assert hasattr(handle, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True).stdout
    exported = sorted(l.split()[-1] for l in out.splitlines() if " T " in l)
    assert exported == _declared()


def test_python_binding_matches_header():
    import old_fmm_bem_b200 as ob
    assert sorted(ob.EXPORTS) == _declared()


def test_config_defaults(lib):
    import old_fmm_bem_b200 as ob
    l = ob.load()
    cfg = ob._Config()
    assert l.fmmb_config_init(ctypes.byref(cfg)) == 0
    assert (cfg.kernel, cfg.p, cfg.lmax, cfg.precision, cfg.semantics, cfg.nrhs) == (0, 8, 3, 0, 0, 1)
    assert l.fmmb_config_init(None) != 0
