"""old_fmm_bem_b200 -- B200-native FMM matvec behind the reference's fmm() interface.

The product is the C-ABI library ``lib/libfmmb.so`` (declared in
``include/fmmb.h``).  This module is the thin host-side binding over it:

* :class:`Plan` -- one configured FMM (kernel, order, depth, precision,
  semantics) with a geometry; ``evaluate`` is one matvec.
* :func:`fmm` / :func:`G_dir` / :func:`Gni_dir` / :func:`Gnj_dir` -- the
  reference's entry points (fmm/fmm.cxx:29, kernel/G_dir.cxx:6,
  kernel/Gni_dir.cxx:6, kernel/Gnj_dir.cxx:6) with the particle arrays passed
  explicitly instead of through globals.

Arrays may be numpy arrays (host) or torch CUDA tensors (device); the library
decides from the pointer.  There is no CPU fallback: without the built library
and a CUDA device every call raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

__all__ = ["Plan", "FMMError", "fmm", "G_dir", "Gni_dir", "Gnj_dir", "lib_path", "load",
           "LAPLACE_G", "LAPLACE_GNI", "LAPLACE_GNJ", "YUKAWA", "HELMHOLTZ_G", "FP64", "MIXED", "SEM_REFERENCE", "SEM_ACCURATE"]

HERE = os.path.dirname(os.path.abspath(__file__))
LAPLACE_G, LAPLACE_GNI, LAPLACE_GNJ = 0, 1, 2
YUKAWA = 10
HELMHOLTZ_G = 20
FP64, MIXED = 0, 1
SEM_REFERENCE, SEM_ACCURATE = 0, 1
EXPORTS = ["fmmb_config_init", "fmmb_plan_create", "fmmb_plan_destroy", "fmmb_set_stream", "fmmb_set_geometry",
           "fmmb_evaluate", "fmmb_evaluate_f64", "fmmb_direct_f64", "fmmb_get_tree_size", "fmmb_get_tree",
           "fmmb_get_expansion_size", "fmmb_get_expansions", "fmmb_get_timings", "fmmb_get_stats",
           "fmmb_last_error", "fmmb_direct_static", "fmmb_autotune_lmax", "fmmb_evaluate_transpose",
           "fmmb_evaluate_transpose_f64", "fmmb_position_grad", "fmmb_set_geometry_batch", "fmmb_gmres_config_init",
           "fmmb_gmres", "fmmb_autotune_lmax_batch", "fmmb_gpu_p2p",
           "fmmb_gpu_p2m", "fmmb_gpu_l2p", "fmmb_gpu_m2l", "fmmb_get_setup_times", "fmmb_set_overlap", "fmmb_adjoint_f64",
           "fmmb_autotune_order"]


def lib_path() -> str:
    return os.path.join(HERE, "lib", "libfmmb.so")


class FMMError(RuntimeError):
    pass


class _Config(ctypes.Structure):
    _fields_ = [("kernel", ctypes.c_int), ("p", ctypes.c_int), ("lmax", ctypes.c_int), ("precision", ctypes.c_int),
                ("semantics", ctypes.c_int), ("eps2", ctypes.c_double), ("exclude_self", ctypes.c_int),
                ("nrhs", ctypes.c_int), ("wavenumber", ctypes.c_double)]


class _GmresConfig(ctypes.Structure):
    _fields_ = [("restart", ctypes.c_int), ("max_iter", ctypes.c_int), ("rtol", ctypes.c_double),
                ("diag", ctypes.c_double), ("precond", ctypes.c_double)]


_LIB = None
_vp = ctypes.c_void_p


def load():
    """Loads libfmmb.so (raises when it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = lib_path()
    if not os.path.exists(path):
        raise FMMError(f"{path} not built: run `python -m old_fmm_bem_b200.build`")
    lib = ctypes.CDLL(path)
    lib.fmmb_config_init.argtypes = [ctypes.POINTER(_Config)]
    lib.fmmb_plan_create.argtypes = [ctypes.POINTER(_Config), ctypes.POINTER(_vp)]
    lib.fmmb_plan_destroy.argtypes = [_vp]
    lib.fmmb_set_stream.argtypes = [_vp, _vp]
    lib.fmmb_set_geometry.argtypes = [_vp, ctypes.c_int] + [_vp] * 6 + [ctypes.c_int] + [_vp] * 6 + [_vp]
    lib.fmmb_set_geometry_batch.argtypes = [_vp, ctypes.c_int, _vp] + [_vp] * 6 + [_vp] + [_vp] * 6 + [_vp]
    lib.fmmb_gmres_config_init.argtypes = [ctypes.POINTER(_GmresConfig)]
    lib.fmmb_gmres.argtypes = [_vp, ctypes.POINTER(_GmresConfig), _vp, _vp, _vp, _vp, _vp]
    lib.fmmb_evaluate.argtypes = [_vp, _vp, _vp, _vp]
    lib.fmmb_evaluate_f64.argtypes = [_vp, _vp, _vp, _vp]
    lib.fmmb_direct_f64.argtypes = [_vp, _vp, ctypes.c_int, ctypes.c_int, _vp, _vp]
    lib.fmmb_evaluate_transpose.argtypes = [_vp, _vp, _vp, _vp]
    lib.fmmb_evaluate_transpose_f64.argtypes = [_vp, _vp, _vp, _vp]
    lib.fmmb_position_grad.argtypes = [_vp, _vp, _vp, _vp, _vp]
    lib.fmmb_adjoint_f64.argtypes = [_vp] * 7
    lib.fmmb_autotune_lmax.argtypes = [ctypes.POINTER(_Config), ctypes.c_int] + [_vp] * 6 + [ctypes.c_int] + \
        [_vp] * 6 + [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp]
    lib.fmmb_autotune_order.argtypes = [ctypes.POINTER(_Config), ctypes.c_int] + [_vp] * 6 + [ctypes.c_int] + \
        [_vp] * 6 + [_vp, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp]
    lib.fmmb_gpu_p2p.argtypes = [_vp] * 15
    lib.fmmb_gpu_p2m.argtypes = [_vp] * 14
    lib.fmmb_gpu_l2p.argtypes = [_vp] * 14
    lib.fmmb_gpu_m2l.argtypes = [_vp] * 6
    lib.fmmb_autotune_lmax_batch.argtypes = [ctypes.POINTER(_Config), ctypes.c_int, _vp] + [_vp] * 6 + [_vp] + \
        [_vp] * 6 + [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp]
    lib.fmmb_direct_static.argtypes = [ctypes.POINTER(_Config), ctypes.c_int] + [_vp] * 6 + [ctypes.c_int] + \
        [_vp] * 6 + [_vp, _vp, _vp, _vp]
    lib.fmmb_get_tree_size.argtypes = [_vp, ctypes.c_int]
    lib.fmmb_get_tree_size.restype = ctypes.c_long
    lib.fmmb_get_tree.argtypes = [_vp, ctypes.c_int, _vp]
    lib.fmmb_get_expansion_size.argtypes = [_vp, ctypes.c_int]
    lib.fmmb_get_expansion_size.restype = ctypes.c_long
    lib.fmmb_get_expansions.argtypes = [_vp, ctypes.c_int, _vp]
    lib.fmmb_get_timings.argtypes = [_vp, _vp]
    lib.fmmb_get_stats.argtypes = [_vp, _vp]
    lib.fmmb_get_setup_times.argtypes = [_vp, _vp]
    lib.fmmb_set_overlap.argtypes = [_vp, ctypes.c_int]
    lib.fmmb_last_error.restype = ctypes.c_char_p
    _LIB = lib
    return lib


def _check(rc):
    if rc != 0:
        msg = load().fmmb_last_error().decode(errors="replace")
        raise FMMError(f"fmmb error {rc}: {msg}")


def _ptr(a, dtype):
    """Pointer of a numpy array (host) or torch tensor (device or host), after
    checking dtype and contiguity.  None stays None."""
    if a is None:
        return None, None
    if hasattr(a, "data_ptr"):  # torch tensor
        import torch
        want = {np.float32: torch.float32, np.float64: torch.float64, np.int32: torch.int32}[dtype]
        if a.dtype != want or not a.is_contiguous():
            raise FMMError(f"expected a contiguous {want} tensor")
        return a.data_ptr(), a
    arr = np.ascontiguousarray(a, dtype=dtype)
    return arr.ctypes.data, arr


class Plan:
    """One FMM configuration bound to a geometry (include/fmmb.h)."""

    def __init__(self, kernel=LAPLACE_G, p=8, lmax=3, precision=FP64, semantics=SEM_REFERENCE, eps2=0.0,
                 exclude_self=False, nrhs=1, wavenumber=0.0):
        lib = load()
        cfg = _Config()
        lib.fmmb_config_init(ctypes.byref(cfg))
        cfg.kernel, cfg.p, cfg.lmax, cfg.precision = kernel, p, lmax, precision
        cfg.semantics, cfg.eps2, cfg.exclude_self, cfg.nrhs = semantics, eps2, int(exclude_self), nrhs
        cfg.wavenumber = wavenumber
        h = _vp()
        _check(lib.fmmb_plan_create(ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self.kernel, self.p, self.lmax, self.precision, self.semantics, self.nrhs = kernel, p, lmax, precision, semantics, nrhs
        self.ni = self.nj = 0
        self._keep = []

    def close(self):
        if getattr(self, "_h", None):
            load().fmmb_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_stream(self, stream):
        """Queue the plan's work on a cudaStream_t (int handle or torch stream)."""
        h = getattr(stream, "cuda_stream", stream)
        _check(load().fmmb_set_stream(self._h, ctypes.c_void_p(h)))
        self._stream = h

    def _follow_torch(self, *arrays):
        """With torch CUDA tensors among the arguments, queue the plan's work on
        torch's current stream, so that it is ordered after the kernels that
        produced the inputs and before those that read the outputs."""
        if any(getattr(a, "is_cuda", False) for a in arrays):
            import torch
            # torch's default stream is the legacy default stream, handle 0,
            # which fmmb_set_stream reads as "the plan's own": pass
            # cudaStreamLegacy ((cudaStream_t)1) for it instead.
            h = torch.cuda.current_stream().cuda_stream or 1
            if h != getattr(self, "_stream", None):
                self.set_stream(h)

    def set_geometry(self, targets, sources, target_normals=None, source_normals=None, bbox=None):
        """targets/sources: (3, n) float32 (numpy or torch); bbox = (xmin, ymin, zmin, rd)."""
        t = [_ptr(targets[k], np.float32) for k in range(3)]
        s = [_ptr(sources[k], np.float32) for k in range(3)]
        tn = [_ptr(target_normals[k], np.float32) for k in range(3)] if target_normals is not None else [(None, None)] * 3
        sn = [_ptr(source_normals[k], np.float32) for k in range(3)] if source_normals is not None else [(None, None)] * 3
        bb = _ptr(np.asarray(bbox, np.float32), np.float32) if bbox is not None else (None, None)
        ni, nj = len(targets[0]), len(sources[0])
        self._follow_torch(*targets, *sources)
        _check(load().fmmb_set_geometry(self._h, ni, t[0][0], t[1][0], t[2][0], tn[0][0], tn[1][0], tn[2][0], nj,
                                        s[0][0], s[1][0], s[2][0], sn[0][0], sn[1][0], sn[2][0], bb[0]))
        self.ni, self.nj = ni, nj
        self.nprob = 1
        return self

    def set_geometry_batch(self, t_off, targets, s_off, sources, target_normals=None, source_normals=None,
                           bbox=None):
        """Independent problems in one plan (fmmb_set_geometry_batch): problem b
        owns targets[:, t_off[b]:t_off[b+1]] and sources[:, s_off[b]:s_off[b+1]];
        t_off / s_off have nprob + 1 entries."""
        to = np.ascontiguousarray(t_off, np.int32)
        so = np.ascontiguousarray(s_off, np.int32)
        assert len(to) == len(so) and len(to) >= 2
        t = [_ptr(targets[k], np.float32) for k in range(3)]
        s = [_ptr(sources[k], np.float32) for k in range(3)]
        tn = [_ptr(target_normals[k], np.float32) for k in range(3)] if target_normals is not None else [(None, None)] * 3
        sn = [_ptr(source_normals[k], np.float32) for k in range(3)] if source_normals is not None else [(None, None)] * 3
        bb = _ptr(np.asarray(bbox, np.float32), np.float32) if bbox is not None else (None, None)
        self._follow_torch(*targets, *sources)
        _check(load().fmmb_set_geometry_batch(self._h, len(to) - 1, to.ctypes.data, t[0][0], t[1][0], t[2][0],
                                              tn[0][0], tn[1][0], tn[2][0], so.ctypes.data, s[0][0], s[1][0],
                                              s[2][0], sn[0][0], sn[1][0], sn[2][0], bb[0]))
        self.ni, self.nj = int(to[-1]), int(so[-1])
        self.nprob = len(to) - 1
        return self

    def gmres(self, b, x=None, weight=None, *, diag=0.0, precond=1.0, restart=30, max_iter=20, rtol=0.0):
        """Batched GMRES (fmmb_gmres) for  diag*x + K(weight .* x) = b  with
        the left preconditioner precond*I, every (rhs, problem) system at once.
        b, x: (nrhs * n,) float64 (numpy or torch CUDA).  Returns (x, iters,
        resid (nrhs, nprob))."""
        cfg = _GmresConfig()
        load().fmmb_gmres_config_init(ctypes.byref(cfg))
        cfg.restart, cfg.max_iter, cfg.rtol, cfg.diag, cfg.precond = restart, max_iter, rtol, diag, precond
        n = self.ni * self.nrhs
        if x is None:
            x = np.zeros(n)
        bp, bk = _ptr(b, np.float64)
        xp, xk = _ptr(x, np.float64)
        wp, wk = _ptr(weight, np.float32)
        nprob = getattr(self, "nprob", 1)
        resid = np.zeros(self.nrhs * nprob)
        it = ctypes.c_int(0)
        self._follow_torch(b, x, weight)
        _check(load().fmmb_gmres(self._h, ctypes.byref(cfg), wp, bp, xp, ctypes.byref(it), resid.ctypes.data))
        return xk, it.value, resid.reshape(self.nrhs, nprob)

    def _complex_call(self, fn_name, q, n_out, out, f64):
        """Helmholtz calls: complex q (numpy or torch complex64) and complex
        outputs (numpy complex128 / complex64, or torch complex tensors), passed
        to the library as interleaved (re, im) floats / doubles."""
        rt = np.float64 if f64 else np.float32
        if hasattr(q, "data_ptr"):
            import torch
            qr = torch.view_as_real(q.to(torch.complex64).contiguous()).contiguous()
            qp = qr.data_ptr()
        else:
            qr = np.ascontiguousarray(q, np.complex64).view(np.float32)
            qp = qr.ctypes.data
        if out is None:
            out = np.zeros(n_out, np.complex128 if f64 else np.complex64)
        if hasattr(out, "data_ptr"):
            import torch
            want = torch.complex128 if f64 else torch.complex64
            if out.dtype != want or not out.is_contiguous():
                raise FMMError(f"expected a contiguous {want} tensor")
            op_ = torch.view_as_real(out).data_ptr()
        else:
            if out.dtype != (np.complex128 if f64 else np.complex64) or not out.flags.c_contiguous:
                raise FMMError("expected a contiguous complex output array")
            op_ = out.ctypes.data
        self._follow_torch(q, out)
        _check(getattr(load(), fn_name)(self._h, qp, op_, None))
        return out

    def evaluate(self, q, pot=None, grad=None, f64=False):
        """One matvec.  q: (nrhs*nj,) charges.  Returns (pot, grad): grad is the
        gradient of the potential w.r.t. the target position (3 blocks of
        nrhs*ni), computed for LAPLACE_G always and for LAPLACE_GNI /
        LAPLACE_GNJ (normals held fixed, accurate semantics) when a grad array
        is given.  Outputs are numpy unless torch CUDA tensors are given."""
        if self.kernel == HELMHOLTZ_G:  # complex charges -> complex potentials, no gradient
            return self._complex_call("fmmb_evaluate_f64" if f64 else "fmmb_evaluate", q, self.ni * self.nrhs, pot,
                                      f64), None
        dt = np.float64 if f64 else np.float32
        qp, qk = _ptr(q, np.float32)
        ni = self.ni * self.nrhs
        if pot is None:
            pot = np.zeros(ni, dt)
        if grad is None and self.kernel == LAPLACE_G:
            grad = np.zeros(3 * ni, dt)
        pp, pk = _ptr(pot, dt)
        gp, gk = _ptr(grad, dt)
        fn = load().fmmb_evaluate_f64 if f64 else load().fmmb_evaluate
        self._follow_torch(q, pot, grad)
        _check(fn(self._h, qp, pp, gp))
        return pk, gk

    def evaluate_transpose(self, w, out=None, grad=None, f64=False):
        """Charge adjoint A^T w (fmmb_evaluate_transpose): w (nrhs*ni,) ->
        (out (nrhs*nj,), grad (3*nrhs*nj,): the gradient of A^T w w.r.t. the
        source position, for LAPLACE_G always, for the normal-derivative kernels
        when grad is given; else None)."""
        if self.kernel == HELMHOLTZ_G:  # A^T w (no conjugation), complex
            return self._complex_call("fmmb_evaluate_transpose_f64" if f64 else "fmmb_evaluate_transpose", w,
                                      self.nj * self.nrhs, out, f64), None
        dt = np.float64 if f64 else np.float32
        wp, wk = _ptr(w, np.float32)
        nj = self.nj * self.nrhs
        if out is None:
            out = np.zeros(nj, dt)
        if grad is None and self.kernel == LAPLACE_G:
            grad = np.zeros(3 * nj, dt)
        op_, ok = _ptr(out, dt)
        gp, gk = _ptr(grad, dt)
        fn = load().fmmb_evaluate_transpose_f64 if f64 else load().fmmb_evaluate_transpose
        self._follow_torch(w, out, grad)
        _check(fn(self._h, wp, op_, gp))
        return ok, gk

    def position_grad(self, q, w, dxt=None, dxs=None):
        """Position gradients of sum(w * pot) (fmmb_position_grad; Laplace
        kernels, normals held fixed): returns (dxt (3, ni), dxs (3, nj)) in FP64."""
        qp, qk = _ptr(q, np.float32)
        wp, wk = _ptr(w, np.float32)
        if dxt is None:
            dxt = np.zeros(3 * self.ni)
        if dxs is None:
            dxs = np.zeros(3 * self.nj)
        tp, tk = _ptr(dxt, np.float64)
        sp, sk = _ptr(dxs, np.float64)
        self._follow_torch(q, w, dxt, dxs)
        _check(load().fmmb_position_grad(self._h, qp, wp, tp, sp))
        return tk.reshape(3, -1), sk.reshape(3, -1)

    def adjoint(self, q, w, field_t=None, dq=None, dxt=None, dxs=None, *, want_dq=True, want_dxs=False):
        """Backward pass of pot = A q for L = sum(w * pot) (fmmb_adjoint_f64):
        dq = A^T w, dxs = q * grad(A^T w)(x_s) and, when the forward's field
        field_t (3 * ni) is given, dxt = w * field_t.  FP64 outputs (numpy
        unless torch CUDA tensors are given); returns (dq, dxt, dxs), None for
        the ones not asked for."""
        qp, qk = _ptr(q, np.float32) if q is not None else (None, None)
        wp, wk = _ptr(w, np.float32)
        fp, fk = _ptr(field_t, np.float64) if field_t is not None else (None, None)
        if dq is None and want_dq:
            dq = np.zeros(self.nj * self.nrhs)
        if dxs is None and want_dxs:
            dxs = np.zeros(3 * self.nj)
        if dxt is None and field_t is not None:
            dxt = np.zeros(3 * self.ni)
        outs = [(_ptr(a, np.float64) if a is not None else (None, None)) for a in (dq, dxt, dxs)]
        self._follow_torch(q, w, field_t, dq, dxt, dxs)
        _check(load().fmmb_adjoint_f64(self._h, qp, wp, fp, outs[0][0], outs[1][0], outs[2][0]))
        return tuple(o[1] for o in outs)

    def direct(self, q, i0=0, i1=None):
        """FP64 direct sum on the GPU for targets [i0, i1) (caller order):
        (pot, grad (3, i1 - i0)), grad = the gradient w.r.t. the target
        position (normals held fixed)."""
        i1 = self.ni if i1 is None else i1
        if self.kernel == HELMHOLTZ_G:  # complex charges, complex128 potentials
            qr = np.ascontiguousarray(q, np.complex64).view(np.float32)
            pot = np.zeros(i1 - i0, np.complex128)
            _check(load().fmmb_direct_f64(self._h, qr.ctypes.data, i0, i1, pot.ctypes.data, None))
            return pot, None
        qp, qk = _ptr(q, np.float32)
        pot = np.zeros(i1 - i0)
        grad = np.zeros(3 * (i1 - i0))
        self._follow_torch(q)
        _check(load().fmmb_direct_f64(self._h, qp, i0, i1, pot.ctypes.data, grad.ctypes.data))
        return pot, grad.reshape(3, -1)

    def tree(self, kind):
        lib = load()
        n = lib.fmmb_get_tree_size(self._h, kind)
        if n < 0:
            _check(int(n))
        out = np.zeros(max(n, 1), np.int32)
        _check(lib.fmmb_get_tree(self._h, kind, out.ctypes.data))
        return out[:n]

    def expansions(self, which):
        lib = load()
        n = lib.fmmb_get_expansion_size(self._h, which)
        if n < 0:
            _check(int(n))
        out = np.zeros(n)
        _check(lib.fmmb_get_expansions(self._h, which, out.ctypes.data))
        return out.reshape(-1, 2) @ np.array([1.0, 1j])

    def timings(self):
        ms = np.zeros(7, np.float32)
        _check(load().fmmb_get_timings(self._h, ms.ctypes.data))
        return dict(zip(["p2p", "p2m", "m2m", "m2l", "l2l", "l2p", "total"], ms.tolist()))

    def set_overlap(self, on: bool):
        """Overlap the near field with the far field (default).  Off: the
        phases run one after another, so timings() gives each phase's time
        with the GPU to itself; the results do not change."""
        _check(load().fmmb_set_overlap(self._h, 1 if on else 0))

    def setup_times(self):
        """(tree build ms, whole fmmb_set_geometry ms) of the current geometry."""
        o = np.zeros(2)
        _check(load().fmmb_get_setup_times(self._h, o.ctypes.data))
        return float(o[0]), float(o[1])

    def stats(self):
        o = np.zeros(8, np.int64)
        _check(load().fmmb_get_stats(self._h, o.ctypes.data))
        return dict(zip(["ni", "nj", "leaves_i", "leaves_j", "p2p_pairs", "m2l_pairs", "lmax", "launches"], o.tolist()))


def _autotune(kernel, p, precision, semantics, eps2, exclude_self, nrhs, ni, nj, lmin, lmax, run):
    lib = load()
    cfg = _Config()
    lib.fmmb_config_init(ctypes.byref(cfg))
    cfg.kernel, cfg.p, cfg.precision, cfg.semantics = kernel, p, precision, semantics
    cfg.eps2, cfg.exclude_self, cfg.nrhs = eps2, int(exclude_self), nrhs
    best = ctypes.c_int(-1)
    ms = np.zeros(16, np.float32)
    _check(run(lib, cfg, best, ms))
    if lmin <= 0 or lmax <= 0:  # the library chose the range around its estimate
        l = 2
        while l < 10 and max(ni, nj) / 8.0 ** l > 64.0:
            l += 1
        lmin, lmax = max(2, l - 1), min(10, l + 2)
    return best.value, {l: float(ms[l - lmin]) for l in range(lmin, lmax + 1)}


def _sets(targets, sources, target_normals, source_normals, bbox):
    t = [_ptr(targets[k], np.float32) for k in range(3)]
    s = [_ptr(sources[k], np.float32) for k in range(3)]
    tn = [_ptr(target_normals[k], np.float32) for k in range(3)] if target_normals is not None else [(None, None)] * 3
    sn = [_ptr(source_normals[k], np.float32) for k in range(3)] if source_normals is not None else [(None, None)] * 3
    bb = _ptr(np.asarray(bbox, np.float32), np.float32) if bbox is not None else (None, None)
    return [x[0] for x in t], [x[0] for x in tn], [x[0] for x in s], [x[0] for x in sn], bb[0], (t, s, tn, sn, bb)


def autotune_lmax(targets, sources, *, kernel=LAPLACE_G, target_normals=None, source_normals=None, p=8,
                  precision=FP64, semantics=SEM_REFERENCE, eps2=0.0, exclude_self=False, bbox=None, lmin=0, lmax=0,
                  reps=3, nrhs=1):
    """Fastest octree depth for this geometry (fmmb_autotune_lmax); returns
    (best_lmax, {lmax: ms per evaluate})."""
    t, tn, s, sn, bb, keep = _sets(targets, sources, target_normals, source_normals, bbox)
    ni, nj = len(targets[0]), len(sources[0])
    return _autotune(kernel, p, precision, semantics, eps2, exclude_self, nrhs, ni, nj, lmin, lmax,
                     lambda lib, cfg, best, ms: lib.fmmb_autotune_lmax(
                         ctypes.byref(cfg), ni, *t, *tn, nj, *s, *sn, bb, lmin, lmax, reps, ctypes.byref(best),
                         ms.ctypes.data))


def autotune_order(targets, sources, tol, *, kernel=LAPLACE_G, target_normals=None, source_normals=None, p_lo=4,
                   p_hi=16, precision=FP64, semantics=SEM_ACCURATE, eps2=0.0, exclude_self=False, bbox=None,
                   nsample=1024, reps=2):
    """Lowest expansion order in [p_lo, p_hi] whose FMM meets the relative
    error tol against the FP64 direct sum on a sample of targets, with its
    autotuned depth (fmmb_autotune_order).  Returns (p, lmax, rel_err,
    ms_per_evaluate); rel_err > tol when no order in the range meets tol."""
    lib = load()
    t, tn, s, sn, bb, keep = _sets(targets, sources, target_normals, source_normals, bbox)
    ni, nj = len(targets[0]), len(sources[0])
    cfg = _Config()
    lib.fmmb_config_init(ctypes.byref(cfg))
    cfg.kernel, cfg.p, cfg.precision, cfg.semantics = kernel, p_lo, precision, semantics
    cfg.eps2, cfg.exclude_self = eps2, int(exclude_self)
    p, lm, err, ms = ctypes.c_int(-1), ctypes.c_int(-1), ctypes.c_double(0.0), ctypes.c_float(0.0)
    _check(lib.fmmb_autotune_order(ctypes.byref(cfg), ni, *t, *tn, nj, *s, *sn, bb, ctypes.c_double(tol), p_lo, p_hi,
                                   nsample, reps, ctypes.byref(p), ctypes.byref(lm), ctypes.byref(err),
                                   ctypes.byref(ms)))
    return p.value, lm.value, err.value, ms.value


def autotune_lmax_batch(t_off, targets, s_off, sources, *, kernel=LAPLACE_G, target_normals=None,
                        source_normals=None, p=8, precision=FP64, semantics=SEM_REFERENCE, eps2=0.0,
                        exclude_self=False, bbox=None, lmin=0, lmax=0, reps=3, nrhs=1):
    """Fastest depth of a forest plan (fmmb_autotune_lmax_batch)."""
    to = np.ascontiguousarray(t_off, np.int32)
    so = np.ascontiguousarray(s_off, np.int32)
    t, tn, s, sn, bb, keep = _sets(targets, sources, target_normals, source_normals, bbox)
    ni, nj = int(to[-1]), int(so[-1])
    return _autotune(kernel, p, precision, semantics, eps2, exclude_self, nrhs, ni, nj, lmin, lmax,
                     lambda lib, cfg, best, ms: lib.fmmb_autotune_lmax_batch(
                         ctypes.byref(cfg), len(to) - 1, to.ctypes.data, *t, *tn, so.ctypes.data, *s, *sn, bb, lmin,
                         lmax, reps, ctypes.byref(best), ms.ctypes.data))


def fmm(xi, yi, zi, gxi, gyi, gzi, xj, yj, zj, gxj, gyj, gzj, vj, neq, *, lmax, xmin, ymin, zmin, rd, p=8,
        precision=FP64, semantics=SEM_REFERENCE):
    """The reference's fmm(mi, mj, neq) (fmm/fmm.cxx:29-152) with explicit arrays.

    neq 0: returns (vi, gxi, gyi, gzi) -- potential and gradient of Laplace G;
    neq 1: returns vi for Gni (gxi.. are the target normals);
    neq 2: returns vi for Gnj (gxj.. are the source normals).
    Arrays in caller order (no sorti/sortj needed)."""
    with Plan(kernel=neq, p=p, lmax=lmax, precision=precision, semantics=semantics) as pl:
        pl.set_geometry((xi, yi, zi), (xj, yj, zj), (gxi, gyi, gzi) if neq == 1 else None,
                        (gxj, gyj, gzj) if neq == 2 else None, bbox=(xmin, ymin, zmin, rd))
        pot, grad = pl.evaluate(vj)
        if neq == 0:
            g = grad.reshape(3, -1)
            return pot, g[0], g[1], g[2]
        return pot


def _direct(neq, xi, yi, zi, gxi, gyi, gzi, xj, yj, zj, gxj, gyj, gzj, vj, semantics=SEM_REFERENCE):
    with Plan(kernel=neq, semantics=semantics, lmax=2) as pl:
        pl.set_geometry((xi, yi, zi), (xj, yj, zj), (gxi, gyi, gzi) if neq == 1 else None,
                        (gxj, gyj, gzj) if neq == 2 else None)
        return pl.direct(vj)


def G_dir(xi, yi, zi, xj, yj, zj, vj, semantics=SEM_REFERENCE):
    """kernel/G_dir.cxx:6-30: potential and gradient by direct summation (FP64)."""
    return _direct(LAPLACE_G, xi, yi, zi, None, None, None, xj, yj, zj, None, None, None, vj, semantics)


def Gni_dir(xi, yi, zi, gxi, gyi, gzi, xj, yj, zj, vj, semantics=SEM_REFERENCE):
    """kernel/Gni_dir.cxx:6-21 (target normals gxi..)."""
    return _direct(LAPLACE_GNI, xi, yi, zi, gxi, gyi, gzi, xj, yj, zj, None, None, None, vj, semantics)[0]


def Gnj_dir(xi, yi, zi, xj, yj, zj, gxj, gyj, gzj, vj, semantics=SEM_REFERENCE):
    """kernel/Gnj_dir.cxx:6-21 (source normals gxj..)."""
    return _direct(LAPLACE_GNJ, xi, yi, zi, None, None, None, xj, yj, zj, gxj, gyj, gzj, vj, semantics)[0]
