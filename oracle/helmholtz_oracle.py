"""FP64 Helmholtz and Yukawa direct sums in numpy -- TEST INFRASTRUCTURE ONLY.

The checker of the FMMB_HELMHOLTZ_G kernel: phi_i = sum_j q_j e^{ik r_ij} /
(4 pi r_ij), zero-distance pairs skipped.  The reference has no oscillatory
Helmholtz kernel (its kernel/Helmholtz_*.cxx is the Yukawa kernel), so parity
is unpinned: this is the kernel's definition evaluated directly, in chunks.

Only tests/ and bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import numpy as np


def direct(xt, xs, q, k, chunk=512):
    """xt (3, ni), xs (3, nj) positions (float32 or float64), q (nj,) complex."""
    xt = np.asarray(xt, np.float64)
    xs = np.asarray(xs, np.float64)
    q = np.asarray(q, np.complex128)
    out = np.zeros(xt.shape[1], np.complex128)
    for i0 in range(0, xt.shape[1], chunk):
        d = xt[:, i0:i0 + chunk, None] - xs[:, None, :]
        r = np.sqrt(np.einsum("kij,kij->ij", d, d))
        zero = r == 0
        r[zero] = 1.0
        g = np.exp(1j * k * r) / (4 * np.pi * r)
        g[zero] = 0.0
        out[i0:i0 + chunk] = g @ q
    return out


def sphere_points(n, seed):
    """n points uniform on the unit sphere (normalised Gaussian vectors) and
    complex charges with real and imaginary parts U[-1, 1]."""
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((3, n))
    v /= np.linalg.norm(v, axis=0)
    q = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    return v.astype(np.float32), q.astype(np.complex64)


def yukawa_direct(xt, xs, q, lam, eps2=0.0, exclude_self=True, chunk=512):
    """The reference's Yukawa kernel (kernel/Helmholtz_G_dir.cxx:15-16):
    sum_j q_j (pi/2) e^{-lam r} / (lam r), r = sqrt(|x_i - x_j|^2 + eps2),
    zero-distance pairs skipped when exclude_self."""
    xt = np.asarray(xt, np.float64)
    xs = np.asarray(xs, np.float64)
    q = np.asarray(q, np.float64)
    out = np.zeros(xt.shape[1])
    for i0 in range(0, xt.shape[1], chunk):
        d = xt[:, i0:i0 + chunk, None] - xs[:, None, :]
        d2 = np.einsum("kij,kij->ij", d, d)
        skip = (d2 == 0) if exclude_self else np.zeros_like(d2, bool)
        r = np.sqrt(d2 + eps2)
        r[skip] = 1.0
        g = 0.5 * np.pi * np.exp(-lam * r) / (lam * r)
        g[skip] = 0.0
        out[i0:i0 + chunk] = g @ q
    return out
