"""Differentiable FMM matvec: a hand-written adjoint behind torch.autograd.

    op = FMMOperator(x_t, x_s, kernel=LAPLACE_G, p=10, lmax=5)   # trees built once
    pot = op(q)                                                 # differentiable
    pot = fmm_potential(x_t, x_s, q, ...)                       # one-shot form

forward: one FMM matvec through the C ABI (libfmmb.so).

backward, for L = sum_i w_i pot_i with w = dL/dpot:
* charges: dL/dq = A^T w, the transposed FMM (targets and sources swapped):
    G   is symmetric:       A^T w = G-FMM(targets = x_s, sources = x_t, charges w)
    Gni (target normals):   A^T w = -Gnj-FMM(targets = x_s, sources = x_t with normals n_t)
    Gnj (source normals):   A^T w = -Gni-FMM(targets = x_s with normals n_s, sources = x_t)
  since d/dx_j G(x_i - x_j) = -d/dx_i G(x_i - x_j).
* positions: dL/dx_t = w * grad_t(A q) and dL/dx_s = q * grad_t(A^T w), grad_t
  the gradient of a matvec's output w.r.t. its target position with the
  normals held fixed: for G the field; for Gnj the field of the double layer;
  for Gni -H n, H the Hessian of the single-layer potential (the transposed
  matvec swaps the two).  The forward computes grad_t(A q) with the
  potential, the backward one transposed FMM with its gradient (the charge
  adjoint comes with it).  When x_t and x_s are the same tensor autograd adds
  the two contributions.  Normals are constants (no gradient flows to them).

An FMMOperator builds the plan (and, through fmmb_evaluate_transpose, its
transposed plan) once; every call reuses the trees, so the geometry
(positions, normals) must stay as it was at construction.  Expansions are
recomputed by each matvec, nothing of size N*P is stored between the passes.
"""
from __future__ import annotations

import torch

from . import FP64, LAPLACE_G, LAPLACE_GNI, LAPLACE_GNJ, MIXED, SEM_ACCURATE, Plan

__all__ = ["FMMOperator", "fmm_potential", "FMMFunction"]

def _col(t):
    return [t[k].contiguous() for k in range(3)]


def _f32(t):
    return t.detach().to(torch.float32).contiguous() if t is not None else None


class FMMOperator:
    """Forward and transposed FMM plans over fixed positions x_t (3, ni) and
    x_s (3, nj) (CUDA tensors), with normals n_t / n_s for Gni / Gnj."""

    def __init__(self, x_t, x_s, *, kernel=LAPLACE_G, n_t=None, n_s=None, p=10, lmax=4, precision=MIXED,
                 semantics=SEM_ACCURATE, eps2=0.0, exclude_self=True, bbox=None):
        self.kernel = kernel
        self.x_t, self.x_s = x_t, x_s
        xt, xs, nt, ns = _f32(x_t), _f32(x_s), _f32(n_t), _f32(n_s)
        self.ni, self.nj = xt.shape[1], xs.shape[1]
        kw = dict(p=p, lmax=lmax, precision=precision, semantics=semantics, eps2=eps2, exclude_self=exclude_self)
        self.plan = Plan(kernel=kernel, **kw)
        self.plan.set_geometry(_col(xt), _col(xs), _col(nt) if kernel == LAPLACE_GNI else None,
                               _col(ns) if kernel == LAPLACE_GNJ else None, bbox=bbox)

    def __call__(self, q):
        """Potential at the targets (FP64 accumulation, returned in q's dtype);
        differentiable w.r.t. q and the position tensors given at construction
        (for Gni / Gnj in accurate semantics)."""
        return FMMFunction.apply(q, self.x_t, self.x_s, self)

    def close(self):
        self.plan.close()


class FMMFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, q, x_t, x_s, op):
        qd = q.detach().to(torch.float32).contiguous()
        pot = torch.empty(op.ni, dtype=torch.float64, device=q.device)  # every entry is written
        want_field = x_t.requires_grad
        grad = torch.empty(3 * op.ni, dtype=torch.float64, device=q.device) if want_field else None
        op.plan.evaluate(qd, pot, grad, f64=True)
        ctx.op = op
        ctx.save_for_backward(qd)
        ctx.field = grad.view(3, op.ni) if grad is not None else None
        ctx.needs = (x_t.requires_grad, x_s.requires_grad)
        return pot.to(q.dtype)

    @staticmethod
    def backward(ctx, w):
        (qd,) = ctx.saved_tensors
        op = ctx.op
        wd = w.detach().to(torch.float32).contiguous()
        # one library call (fmmb_adjoint_f64): the transposed FMM (targets x_s,
        # sources x_t, charges w; the sign of the normal-derivative kernels is
        # applied there; on one point set the plan itself for G) and the
        # weighting of the two fields
        f64 = dict(dtype=torch.float64, device=w.device)
        want_q = ctx.needs_input_grad[0]
        want_xt, want_xs = ctx.needs
        dq = torch.empty(op.nj, **f64) if want_q else None
        dxt = torch.empty(3 * op.ni, **f64) if want_xt else None
        dxs = torch.empty(3 * op.nj, **f64) if want_xs else None
        if want_q or want_xt or want_xs:
            op.plan.adjoint(qd, wd, ctx.field.reshape(-1) if want_xt else None, dq, dxt, dxs,
                            want_dq=want_q, want_dxs=want_xs)
        return (dq.to(w.dtype) if dq is not None else None,
                dxt.view(3, op.ni).to(w.dtype) if dxt is not None else None,
                dxs.view(3, op.nj).to(w.dtype) if dxs is not None else None, None)


def fmm_potential(x_t, x_s, q, *, kernel=LAPLACE_G, n_t=None, n_s=None, p=10, lmax=4, precision=MIXED,
                  semantics=SEM_ACCURATE, eps2=0.0, exclude_self=True, bbox=None):
    """Differentiable FMM potential at targets x_t (3, ni) of charges q (nj,)
    at sources x_s (3, nj), all CUDA tensors (builds the trees for this call;
    use FMMOperator to reuse them).  Gradients flow to q and to x_t / x_s."""
    op = FMMOperator(x_t, x_s, kernel=kernel, n_t=n_t, n_s=n_s, p=p, lmax=lmax, precision=precision,
                     semantics=semantics, eps2=eps2, exclude_self=exclude_self, bbox=bbox)
    return op(q)
