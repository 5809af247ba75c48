"""Reverse-mode differentiation of the pass at fixed topology.

:class:`FMMAccelerations` is a ``torch.autograd.Function`` whose forward is the
whole evaluation pass on live positions / masses (COM centres included) and
whose backward is the hand-written adjoint kernels (``Pass.vjp``) -- the torch
counterpart of the reference's ``jax.custom_vjp`` around
``differentiable_accelerations`` (runtime/fmm_evaluate.py:542-731, :1175-1250).

Memory policy: the forward's node coefficients (centres, multipoles, locals:
num_nodes x (2 stride + 4) floats) are kept for the backward when they fit in
``keep_bytes``; above that the backward recomputes them from the saved inputs.
"""

from __future__ import annotations

import torch

from .engine import Pass

DEFAULT_KEEP_BYTES = 1 << 30


class FMMAccelerations(torch.autograd.Function):
    @staticmethod
    def forward(ctx, positions: torch.Tensor, masses: torch.Tensor, pass_: Pass, keep_bytes: int = DEFAULT_KEEP_BYTES):
        n = pass_.dt.topo.num_particles
        pass_.load_particles(positions.detach(), masses.detach())
        pass_.run(cascade=True)  # the backward reads every node's complete local
        acc = torch.empty((n, 3), device=pass_.dt.device, dtype=torch.float32)
        pass_.unsort(acc, None)
        ws = pass_.ws
        coeff_bytes = 4 * (ws.centers.numel() + ws.mult.numel() + ws.locals.numel())
        ctx.kept = None
        if coeff_bytes <= keep_bytes:
            ctx.kept = (ws.centers.clone(), ws.mult.clone(), ws.locals.clone())
        ctx.pass_ = pass_
        ctx.save_for_backward(positions.detach(), masses.detach())
        return acc.to(positions.dtype)

    @staticmethod
    def backward(ctx, grad_acc: torch.Tensor):
        positions, masses = ctx.saved_tensors
        ps: Pass = ctx.pass_
        n = ps.dt.topo.num_particles
        ps.load_particles(positions, masses)
        if ctx.kept is not None:
            ps.ws.centers.copy_(ctx.kept[0])
            ps.ws.mult.copy_(ctx.kept[1])
            ps.ws.locals.copy_(ctx.kept[2])
        gx = torch.empty((n, 3), device=ps.dt.device, dtype=torch.float32)
        gm = torch.empty((n,), device=ps.dt.device, dtype=torch.float32)
        ps.vjp(grad_acc.contiguous(), gx, gm, recompute=ctx.kept is None)
        return gx.to(positions.dtype), gm.to(masses.dtype), None, None


def fmm_accelerations(positions: torch.Tensor, masses: torch.Tensor, pass_: Pass,
                      keep_bytes: int = DEFAULT_KEEP_BYTES) -> torch.Tensor:
    """Accelerations (N,3) in input order, differentiable w.r.t. both inputs."""
    return FMMAccelerations.apply(positions, masses, pass_, keep_bytes)
