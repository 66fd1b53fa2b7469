"""Thin ``torch.autograd.Function`` wrappers over the adjoint derivatives.

They exist for gradient checks (``torch.autograd.gradcheck`` runs central
finite differences against the adjoint): the forward pass calls the C ABI
through :mod:`scft_string_b200` and the backward pass returns the derivative
the adjoint already computed.  Nothing in the solver depends on torch.

* :class:`LnQOfBox` -- lnQ of one replica at fixed fields as a function of the
  box lengths (L_x, L_y, L_z); backward = d lnQ/dL from ``scft_stress`` or,
  with ``K > 0``, from the checkpointed ``scft_stress_ckpt``.
* :class:`SaddleFreeEnergy` -- the free energy per chain at the saddle point
  (fields re-converged by Anderson mixing from a start field) as a function of
  (L_x, L_y, L_z, chiN); backward = (dF/dL, dF/dchiN) = (-d lnQ/dL,
  1/4 - <W-^2>/chiN^2), exact at the saddle point.
"""
from __future__ import annotations

import numpy as np
import torch

from . import Context


def _free_energy(ctx: Context, ii: int, chi: float) -> float:
    """F = -lnQ + <chi pA pB - wA pA - wB pB> (scft.cu:823-826)."""
    M = ctx.M
    ctx.props(ii)
    conc, lnQ, _ = ctx.get_conc(ii)
    W = ctx.get_fields(ii)
    pA, pB = conc[:M], conc[M:2 * M]
    wa, wb = W[:M] + W[M:], W[M:] - W[:M]
    return float(-lnQ + np.mean(chi * pA * pB - wa * pA - wb * pB))


class LnQOfBox(torch.autograd.Function):
    @staticmethod
    def forward(fctx, L, ctx: Context, ii: int = 0, K: int = 0):
        ctx.set_box(L.detach().cpu().double().numpy())
        if K > 0:
            dlnq, _, _ = ctx.stress_ckpt(ii, K)
        else:
            dlnq, _ = ctx.stress(ii)
        ctx.props(ii)
        lnQ = ctx.get_conc(ii)[1]
        fctx.save_for_backward(torch.as_tensor(dlnq, dtype=L.dtype, device=L.device))
        return torch.as_tensor(lnQ, dtype=L.dtype, device=L.device)

    @staticmethod
    def backward(fctx, g):
        (d,) = fctx.saved_tensors
        return g * d, None, None, None


class SaddleFreeEnergy(torch.autograd.Function):
    @staticmethod
    def forward(fctx, p, make_ctx, w0, tol: float = 1e-10):
        """p = (L_x, L_y, L_z, chiN); make_ctx(D, chi) -> one-replica Context;
        w0 = start fields [W-, W+] (2M float64)."""
        v = p.detach().cpu().double().numpy()
        D, chi = v[:3], float(v[3])
        ctx = make_ctx(D, chi)
        ctx.set_fields_2m(0, np.ascontiguousarray(w0, np.float64))
        _, err = ctx.anderson_solve(0, maxIter=4000, tol=tol, nhist=12, lam=0.1)
        if not err <= 10 * tol:
            raise RuntimeError(f"saddle point not reached: residual {err:g}")
        F = _free_energy(ctx, 0, chi)
        _, dF = ctx.stress(0)
        grad = np.concatenate([dF, [ctx.dF_dchi(0)]])
        ctx.close()
        fctx.save_for_backward(torch.as_tensor(grad, dtype=p.dtype, device=p.device))
        return torch.as_tensor(F, dtype=p.dtype, device=p.device)

    @staticmethod
    def backward(fctx, g):
        (d,) = fctx.saved_tensors
        return g * d, None, None, None
