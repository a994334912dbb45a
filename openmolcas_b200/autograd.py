"""The two-electron energy as a differentiable torch function.

    E(R, C) = 1/2 tr(D J) - 1/4 tr(D K),   D = C C^T

Forward: ERI Cholesky decomposition at the nuclear coordinates R
(Cho_Drv, algorithm 4) and the Cholesky J/K build (CHO_LK_SCF) for the density
factor C.  Backward: the hand-written adjoint -- the two-electron gradient
kernel (Drvg1: derivative Rys integrals recomputed tile by tile, contracted
with the 2-PDM of D) for dE/dR, and dE/dC = 2 (J - K/2) C for the factor
(J and K are linear and symmetric in D).  The gradient kernel differentiates
the exact-integral energy; the forward energy carries the decomposition
error (ThrCom), so finite differences of the forward agree with the backward
to that level.
"""
from __future__ import annotations

import torch

from .molgpu import MolGpu


class JKEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coords, C, mol, thrcom=1e-8, cutint=1e-14, precision=MolGpu.PREC_FP64, device=0):
        m = mol.at(coords.detach().to("cpu", torch.float64).numpy())
        g = MolGpu(m, device)
        g.cho_drv(thrcom=thrcom)
        dev = f"cuda:{device}"
        Cd = C.detach().to(dev, torch.float64)
        J, K = g.cho_jk(Cd, precision=precision)
        D = Cd @ Cd.t()
        E = 0.5 * (D * J).sum() - 0.25 * (D * K).sum()
        ctx.save_for_backward(Cd, J, K)
        ctx.g, ctx.D, ctx.cutint = g, D, cutint
        ctx.coords_meta = (coords.device, coords.dtype)
        ctx.c_meta = (C.device, C.dtype)
        return E.to(coords.device, coords.dtype)

    @staticmethod
    def backward(ctx, gE):
        Cd, J, K = ctx.saved_tensors
        dR = dC = None
        scale = gE.to(Cd.device, torch.float64)
        if ctx.needs_input_grad[0]:
            dR = (ctx.g.drvg1(ctx.D, cutint=ctx.cutint) * scale).to(*ctx.coords_meta)
        if ctx.needs_input_grad[1]:
            dC = (2.0 * (J - 0.5 * K) @ Cd * scale).to(*ctx.c_meta)
        return dR, dC, None, None, None, None, None


def jk_energy(coords, C, mol, **kw):
    """E = 1/2 tr(DJ) - 1/4 tr(DK) for D = C C^T at `coords`, differentiable in
    coords (through the gradient kernel) and in C."""
    return JKEnergy.apply(coords, C, mol, kw.get("thrcom", 1e-8), kw.get("cutint", 1e-14),
                          kw.get("precision", MolGpu.PREC_FP64), kw.get("device", 0))
