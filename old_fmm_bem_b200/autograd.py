"""Differentiable FMM matvec: a hand-written adjoint behind torch.autograd.

    pot = fmm_potential(x_t, x_s, q, kernel=LAPLACE_G, p=10, lmax=5, ...)

forward: one FMM matvec through the C ABI (libfmmb.so).

backward, for L = sum_i w_i pot_i with w = dL/dpot:
* charges: dL/dq = A^T w, the transposed FMM (targets and sources swapped):
    G   is symmetric:       A^T w = G-FMM(targets = x_s, sources = x_t, charges w)
    Gni (target normals):   A^T w = -Gnj-FMM(targets = x_s, sources = x_t with normals n_t)
    Gnj (source normals):   A^T w = -Gni-FMM(targets = x_s with normals n_s, sources = x_t)
  since d/dx_j G(x_i - x_j) = -d/dx_i G(x_i - x_j).
* positions (Laplace G): dL/dx_t = w * grad(pot)(x_t) (the forward FMM's field) and
  dL/dx_s = q * grad(psi)(x_s) with psi = G-FMM(targets x_s, sources x_t,
  charges w) -- the same transposed FMM as the charge adjoint, with its field.
  So a backward costs one FMM with gradient.  When x_t and x_s are the same
  tensor autograd adds the two contributions.
  (Position gradients of the normal-derivative kernels need second
  derivatives of the kernel and are not provided: their positions must not
  require grad.)

Both FMMs keep their trees: the forward plan and the transposed plan are built
in forward and reused by backward (the expansions are recomputed, nothing of
size N*P is stored between the passes).
"""
from __future__ import annotations

import torch

from . import FP64, LAPLACE_G, LAPLACE_GNI, LAPLACE_GNJ, MIXED, SEM_ACCURATE, Plan

__all__ = ["fmm_potential", "FMMFunction"]


def _col(t):
    return [t[k].contiguous() for k in range(3)]


class FMMFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, q, x_t, x_s, n_t, n_s, opts):
        kernel = opts["kernel"]
        dev = q.device
        qd = q.detach().to(torch.float32).contiguous()
        xt, xs = x_t.detach().to(torch.float32).contiguous(), x_s.detach().to(torch.float32).contiguous()
        nt = n_t.detach().to(torch.float32).contiguous() if n_t is not None else None
        ns = n_s.detach().to(torch.float32).contiguous() if n_s is not None else None
        bbox = opts.get("bbox")
        plan = Plan(kernel=kernel, p=opts["p"], lmax=opts["lmax"], precision=opts["precision"],
                    semantics=opts["semantics"], eps2=opts["eps2"], exclude_self=opts["exclude_self"])
        plan.set_geometry(_col(xt), _col(xs), _col(nt) if kernel == LAPLACE_GNI else None,
                          _col(ns) if kernel == LAPLACE_GNJ else None, bbox=bbox)
        ni = xt.shape[1]
        pot = torch.zeros(ni, dtype=torch.float64, device=dev)
        grad = torch.zeros(3 * ni, dtype=torch.float64, device=dev) if kernel == LAPLACE_G else None
        plan.evaluate(qd, pot, grad, f64=True)
        ctx.plan = plan
        ctx.opts = opts
        ctx.geom = (xt, xs, nt, ns)
        ctx.save_for_backward(qd)
        ctx.field = grad.view(3, ni) if grad is not None else None
        ctx.needs = (x_t.requires_grad, x_s.requires_grad)
        if kernel != LAPLACE_G and (x_t.requires_grad or x_s.requires_grad):
            raise ValueError("position gradients are provided for the Laplace G kernel only")
        return pot.to(q.dtype)

    @staticmethod
    def backward(ctx, w):
        (qd,) = ctx.saved_tensors
        opts = ctx.opts
        kernel = opts["kernel"]
        xt, xs, nt, ns = ctx.geom
        wd = w.detach().to(torch.float32).contiguous()
        # transposed FMM: targets x_s, sources x_t, charges w
        tkernel = {LAPLACE_G: LAPLACE_G, LAPLACE_GNI: LAPLACE_GNJ, LAPLACE_GNJ: LAPLACE_GNI}[kernel]
        sign = 1.0 if kernel == LAPLACE_G else -1.0
        plan_t = Plan(kernel=tkernel, p=opts["p"], lmax=opts["lmax"], precision=opts["precision"],
                      semantics=opts["semantics"], eps2=opts["eps2"], exclude_self=opts["exclude_self"])
        plan_t.set_geometry(_col(xs), _col(xt), _col(ns) if tkernel == LAPLACE_GNI else None,
                            _col(nt) if tkernel == LAPLACE_GNJ else None, bbox=opts.get("bbox"))
        nj = xs.shape[1]
        adj = torch.zeros(nj, dtype=torch.float64, device=w.device)
        field = torch.zeros(3 * nj, dtype=torch.float64, device=w.device) if tkernel == LAPLACE_G else None
        plan_t.evaluate(wd, adj, field, f64=True)
        plan_t.close()
        dq = (sign * adj).to(w.dtype)
        dxt = dxs = None
        if kernel == LAPLACE_G:
            if ctx.needs[0]:
                dxt = (w.to(torch.float64) * ctx.field).to(w.dtype)
            if ctx.needs[1]:
                dxs = (qd.to(torch.float64) * field.view(3, nj)).to(w.dtype)
        ctx.plan.close()
        return dq, dxt, dxs, None, None, None


def fmm_potential(x_t, x_s, q, *, kernel=LAPLACE_G, n_t=None, n_s=None, p=10, lmax=4, precision=MIXED,
                  semantics=SEM_ACCURATE, eps2=0.0, exclude_self=True, bbox=None):
    """Differentiable FMM potential at targets x_t (3, ni) of charges q (nj,)
    at sources x_s (3, nj), all CUDA tensors.  Gradients flow to q (all
    kernels) and to x_t / x_s (Laplace G)."""
    opts = dict(kernel=kernel, p=p, lmax=lmax, precision=precision, semantics=semantics, eps2=eps2,
                exclude_self=exclude_self, bbox=bbox)
    return FMMFunction.apply(q, x_t, x_s, n_t, n_s, opts)
