"""PyTorch operator surface of the two-electron path: ``torch.ops.molgpu.*``.

The reference has no in-process Python API (pymolcas only launches the
Fortran programs, Tools/pymolcas/molcas_wrapper.py), so these operators are
the Python-side drop-in for its driver boundaries, each a thin call into the
C ABI of ``libmolgpu.so`` through a ``MolGpu`` handle:

    molgpu::eri_batch(handle, quartets)          Drv2El/Eval_IJKL batch -> (blocks, offsets)
    molgpu::cholesky(handle, thrcom, span, minqual, maxqual)
                                                 Cho_Drv -> [nrs, M, npass]
    molgpu::jk(handle, C, precision)             CHO_LK_SCF -> (J, K)
    molgpu::jk_energy(handle, C, precision)      E = 1/2 tr(DJ) - 1/4 tr(DK), D = C C^T,
                                                 differentiable in C (dE/dC = 2 (J - K/2) C)

A handle is the integer returned by ``register(MolGpu)``; the basis and the
Cholesky vectors live on the device inside it.  The nuclear-coordinate
derivative goes through ``autograd.jk_energy`` (the gradient kernel).
"""
from __future__ import annotations

import numpy as np
import torch

from .molgpu import MolGpu, MolGpuError

_handles: dict[int, MolGpu] = {}


def register(g: MolGpu) -> int:
    """Make a MolGpu usable from the operators; returns its handle number."""
    h = id(g) & 0x7FFFFFFF
    while h in _handles and _handles[h] is not g:
        h = (h + 1) & 0x7FFFFFFF
    _handles[h] = g
    return h


def unregister(h: int) -> None:
    _handles.pop(int(h), None)


def _get(h: int) -> MolGpu:
    try:
        return _handles[int(h)]
    except KeyError:
        raise MolGpuError(f"molgpu: unknown handle {h} (call torch_ops.register)") from None


@torch.library.custom_op("molgpu::eri_batch", mutates_args=())
def eri_batch(handle: int, quartets: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
    """Shell-quartet ERI blocks in Eval_IJKL layout for an (nq, 4) int32 list of
    canonical quartets (i >= j, k >= l); returns (device FP64 blocks, int64
    offsets[nq + 1])."""
    g = _get(handle)
    q = np.ascontiguousarray(quartets.detach().to("cpu", torch.int32).numpy())
    out, off = g.eri_quartets(q)
    return out, torch.from_numpy(off.astype(np.int64))


@eri_batch.register_fake
def _(handle, quartets):
    n = quartets.shape[0]
    return (torch.empty(0, dtype=torch.float64, device="cuda"), torch.empty(n + 1, dtype=torch.int64))


@torch.library.custom_op("molgpu::cholesky", mutates_args=())
def cholesky(handle: int, thrcom: float, span: float, minqual: int, maxqual: int) -> torch.Tensor:
    """Cho_Drv (algorithm 4) on the handle's basis; returns int64 [nrs, M, npass]."""
    info = _get(handle).cho_drv(thrcom=thrcom, span=span, minqual=minqual, maxqual=maxqual)
    return torch.tensor([info["nrs"], info["M"], info["npass"]], dtype=torch.int64)


@cholesky.register_fake
def _(handle, thrcom, span, minqual, maxqual):
    return torch.empty(3, dtype=torch.int64)


@torch.library.custom_op("molgpu::jk", mutates_args=())
def jk(handle: int, C: torch.Tensor, precision: int) -> tuple[torch.Tensor, torch.Tensor]:
    """CHO_LK_SCF for D = C C^T (C: nbf x r): (J, K), nbf x nbf FP64 on the device."""
    return _get(handle).cho_jk(C, precision=precision)


@jk.register_fake
def _(handle, C, precision):
    n = C.shape[0]
    return (C.new_empty((n, n), dtype=torch.float64), C.new_empty((n, n), dtype=torch.float64))


@torch.library.custom_op("molgpu::jk_energy", mutates_args=())
def jk_energy(handle: int, C: torch.Tensor, precision: int) -> torch.Tensor:
    """E = 1/2 tr(D J) - 1/4 tr(D K) for D = C C^T (0-d FP64 tensor)."""
    g = _get(handle)
    Cd = C.detach().to(f"cuda:{g.device}", torch.float64)
    J, K = g.cho_jk(Cd, precision=precision)
    D = Cd @ Cd.t()
    return (0.5 * (D * J).sum() - 0.25 * (D * K).sum()).to(C.device)


@jk_energy.register_fake
def _(handle, C, precision):
    return C.new_empty((), dtype=torch.float64)


def _jk_energy_setup(ctx, inputs, output):
    handle, C, precision = inputs
    ctx.handle, ctx.precision = handle, precision
    ctx.save_for_backward(C)


def _jk_energy_backward(ctx, gE):
    (C,) = ctx.saved_tensors
    g = _get(ctx.handle)
    Cd = C.detach().to(f"cuda:{g.device}", torch.float64)
    J, K = g.cho_jk(Cd, precision=ctx.precision)
    dC = 2.0 * (J - 0.5 * K) @ Cd * gE.to(Cd.device, torch.float64)
    return None, dC.to(C.device, C.dtype), None


torch.library.register_autograd("molgpu::jk_energy", _jk_energy_backward, setup_context=_jk_energy_setup)
