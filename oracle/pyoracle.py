"""ctypes access to the oracle libraries -- TEST INFRASTRUCTURE ONLY.

Two checkers live under oracle/:

* ``liboracle.so`` -- the CPU restatement of the reference FMM
  (oracle/fmm_oracle.cpp), runtime order p, reference or accurate semantics,
  plus an FP64 direct sum;
* ``_ref/libfmmref_mp<p+1>.so`` -- the reference's own CPU FMM compiled from
  its sources by oracle/Makefile (fmm/fmm.cxx:29 driven the way
  test/test.cxx:106-116 drives it, level-2 neighbour mode fixed).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  The product library never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_fp = ctypes.POINTER(ctypes.c_float)
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
EPS_REF = float(np.float32(1e-6))  # the reference's eps (include/constants.h:34)


class oracle_config(ctypes.Structure):
    _fields_ = [("p", ctypes.c_int), ("lmax", ctypes.c_int), ("neq", ctypes.c_int),
                ("ref_semantics", ctypes.c_int), ("eps2", ctypes.c_double),
                ("exclude_self", ctypes.c_int), ("xmin", ctypes.c_float),
                ("ymin", ctypes.c_float), ("zmin", ctypes.c_float), ("rd", ctypes.c_float)]


def _f(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32).ctypes.data_as(_fp)


_libs: dict = {}


def build():
    """Compile the restatement (and the reference libraries where the reference
    sources are present)."""
    subprocess.run(["make", "-s", "-f", os.path.join(HERE, "Makefile"), "all"], check=True)


def _load(path):
    if path not in _libs:
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -f oracle/Makefile`")
        _libs[path] = ctypes.CDLL(path)
    return _libs[path]


def oracle_lib():
    lib = _load(os.path.join(HERE, "liboracle.so"))
    lib.oracle_fmm.restype = ctypes.c_int
    lib.oracle_fmm.argtypes = [ctypes.POINTER(oracle_config), ctypes.c_int, ctypes.c_int] + [_fp] * 13 + [_dp] * 4
    lib.oracle_direct.restype = ctypes.c_int
    lib.oracle_direct.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int] + [_fp] * 13 + [_dp] * 4
    lib.oracle_record_size.restype = ctypes.c_long
    lib.oracle_record_copy.argtypes = [ctypes.c_int, _ip]
    lib.oracle_expansion_size.restype = ctypes.c_long
    lib.oracle_expansion_copy.argtypes = [ctypes.c_int, _dp]
    return lib


def ref_lib(p, gpu_p2p=False, perf=False):
    """The reference library of order p; gpu_p2p: the p = 8 build whose near
    field runs through the reference's p2pgpu_ callers into libfmmb; perf: the
    build made for timing (same sources, vectorising -march, oracle/Makefile
    target perf)."""
    name = "libfmmref_gpup2p_mp9.so" if gpu_p2p else (f"libfmmref_perf_mp{p + 1}.so" if perf else
                                                       f"libfmmref_mp{p + 1}.so")
    if gpu_p2p:
        assert p == 8, "the p2pgpu_ build is made for mp = 9"
    lib = _load(os.path.join(HERE, "_ref", name))
    lib.ref_fmm.restype = ctypes.c_int
    lib.ref_fmm.argtypes = [ctypes.c_int] * 4 + [ctypes.c_float] * 4 + [ctypes.c_double] + [_fp] * 13 + [_fp] * 4 + [_dp]
    lib.ref_direct.restype = ctypes.c_int
    lib.ref_direct.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] + [_fp] * 13 + [_fp] * 4
    lib.ref_record_size.restype = ctypes.c_long
    lib.ref_record_copy.argtypes = [ctypes.c_int, _ip]
    return lib


def ref_available(p, perf=False):
    return os.path.exists(os.path.join(HERE, "_ref", f"libfmmref_{'perf_' if perf else ''}mp{p + 1}.so"))


def _unpack(t, tn, s, sn, q):
    t = np.ascontiguousarray(t, np.float32)
    s = np.ascontiguousarray(s, np.float32)
    tn = np.zeros_like(t) if tn is None else np.ascontiguousarray(tn, np.float32)
    sn = np.zeros_like(s) if sn is None else np.ascontiguousarray(sn, np.float32)
    q = np.ascontiguousarray(q, np.float32)
    return t, tn, s, sn, q


def oracle_fmm(t, s, q, *, neq=0, p=8, lmax=3, bbox=(0.0, 0.0, 0.0, 1.0), ref_semantics=True,
               eps2=None, exclude_self=False, tn=None, sn=None):
    """Restatement FMM.  t, s: (3, n) float32; returns (pot, grad(3,n) or None)
    in FP64, caller order."""
    lib = oracle_lib()
    t, tn, s, sn, q = _unpack(t, tn, s, sn, q)
    ni, nj = t.shape[1], s.shape[1]
    if eps2 is None:
        eps2 = EPS_REF if ref_semantics else 0.0
    cfg = oracle_config(p, lmax, neq, int(ref_semantics), eps2, int(exclude_self), *[np.float32(b) for b in bbox])
    pot = np.zeros(ni)
    g = np.zeros((3, ni))
    rc = lib.oracle_fmm(ctypes.byref(cfg), ni, nj, _f(t[0]), _f(t[1]), _f(t[2]), _f(tn[0]), _f(tn[1]), _f(tn[2]),
                        _f(s[0]), _f(s[1]), _f(s[2]), _f(sn[0]), _f(sn[1]), _f(sn[2]), _f(q),
                        pot.ctypes.data_as(_dp), g[0].ctypes.data_as(_dp), g[1].ctypes.data_as(_dp),
                        g[2].ctypes.data_as(_dp))
    if rc != 0:
        raise RuntimeError(f"oracle_fmm failed ({rc})")
    return pot, (g if neq == 0 else None)


def oracle_records():
    lib = oracle_lib()
    out = {}
    for k in range(9):
        n = lib.oracle_record_size(k)
        a = np.zeros(max(n, 1), np.int32)
        lib.oracle_record_copy(k, a.ctypes.data_as(_ip))
        out[k] = a[:n]
    return out


def oracle_expansions(which):
    lib = oracle_lib()
    n = lib.oracle_expansion_size(which)
    a = np.zeros(max(n, 1))
    lib.oracle_expansion_copy(which, a.ctypes.data_as(_dp))
    return a[:n].reshape(-1, 2) @ np.array([1.0, 1j])


def direct(t, s, q, *, neq=0, eps2=0.0, exclude_self=True, ref_pi=False, tn=None, sn=None, targets=None):
    """FP64 direct sum at targets[i0:i1] (default all)."""
    lib = oracle_lib()
    t, tn, s, sn, q = _unpack(t, tn, s, sn, q)
    ni, nj = t.shape[1], s.shape[1]
    i0, i1 = (0, ni) if targets is None else targets
    m = i1 - i0
    pot = np.zeros(m)
    g = np.zeros((3, m))
    rc = lib.oracle_direct(neq, eps2, int(exclude_self), int(ref_pi), ni, nj, i0, i1,
                           _f(t[0]), _f(t[1]), _f(t[2]), _f(tn[0]), _f(tn[1]), _f(tn[2]),
                           _f(s[0]), _f(s[1]), _f(s[2]), _f(sn[0]), _f(sn[1]), _f(sn[2]), _f(q),
                           pot.ctypes.data_as(_dp), g[0].ctypes.data_as(_dp), g[1].ctypes.data_as(_dp),
                           g[2].ctypes.data_as(_dp))
    if rc != 0:
        raise RuntimeError("oracle_direct failed")
    return pot, (g if neq == 0 else None)


def ref_fmm(t, s, q, *, neq=0, p=8, lmax=3, bbox=(0.0, 0.0, 0.0, 1.0), tn=None, sn=None, lam=0.0,
            timings=None, gpu_p2p=False, perf=False):
    """The reference's own fmm() (built from its sources).  Returns float32
    (pot, grad) in caller order; the reference computes the gradient for neq 0."""
    lib = ref_lib(p, gpu_p2p, perf)
    t, tn, s, sn, q = _unpack(t, tn, s, sn, q)
    ni, nj = t.shape[1], s.shape[1]
    v = np.zeros(ni, np.float32)
    g = np.zeros((3, ni), np.float32)
    tm = np.zeros(100) if timings is None else timings
    lib.ref_fmm(ni, nj, neq, lmax, *[np.float32(b) for b in bbox], lam,
                _f(t[0]), _f(t[1]), _f(t[2]), _f(tn[0]), _f(tn[1]), _f(tn[2]),
                _f(s[0]), _f(s[1]), _f(s[2]), _f(sn[0]), _f(sn[1]), _f(sn[2]), _f(q),
                v.ctypes.data_as(_fp), g[0].ctypes.data_as(_fp), g[1].ctypes.data_as(_fp), g[2].ctypes.data_as(_fp),
                tm.ctypes.data_as(_dp))
    return v, (g if neq == 0 else None)


def ref_direct(t, s, q, *, neq=0, p=8, lam=0.0, tn=None, sn=None):
    """The reference's own direct sums (kernel/G_dir.cxx, Gni_dir.cxx,
    Gnj_dir.cxx, Helmholtz_G_dir.cxx for neq 10 with screening lam), float32
    outputs in caller order: (pot, grad or None)."""
    lib = ref_lib(p)
    t, tn, s, sn, q = _unpack(t, tn, s, sn, q)
    ni, nj = t.shape[1], s.shape[1]
    v = np.zeros(ni, np.float32)
    g = np.zeros((3, ni), np.float32)
    lib.ref_direct(ni, nj, neq, lam, _f(t[0]), _f(t[1]), _f(t[2]), _f(tn[0]), _f(tn[1]), _f(tn[2]),
                   _f(s[0]), _f(s[1]), _f(s[2]), _f(sn[0]), _f(sn[1]), _f(sn[2]), _f(q),
                   v.ctypes.data_as(_fp), g[0].ctypes.data_as(_fp), g[1].ctypes.data_as(_fp), g[2].ctypes.data_as(_fp))
    return v, (g if neq == 0 else None)


def ref_records(p):
    lib = ref_lib(p)
    out = {}
    for k in range(9):
        n = lib.ref_record_size(k)
        a = np.zeros(max(n, 1), np.int32)
        lib.ref_record_copy(k, a.ctypes.data_as(_ip))
        out[k] = a[:n]
    return out


def parse_lists(stream):
    """Split a list stream [lev, mode, nbi, nbj, counts..., entries...]* into
    [(lev, mode, nbj, [list per target box])]."""
    out = []
    i = 0
    s = list(stream)
    while i < len(s):
        lev, mode, nbi, nbj = s[i:i + 4]
        i += 4
        counts = s[i:i + nbi]
        i += nbi
        lists = []
        for c in counts:
            lists.append(s[i:i + c])
            i += c
        out.append((lev, mode, nbj, lists))
    return out
