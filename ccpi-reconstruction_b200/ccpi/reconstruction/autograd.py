"""Differentiable projector: ``A`` as a ``torch.autograd.Function``.

The forward pass is the library's forward projector (``ccpi_forward``) and
the backward pass is its matched back projector (``ccpi_backward``), the
exact transpose of the same Siddon ray model (Core/src/c2D.cpp:469-625 and
:948-1119 for cone beam, Core/src/p2D.cpp:468-611 and :950-1087 for
parallel beam).  Both run as hand-written CUDA kernels on torch's current
stream; torch only supplies the tensors.

Shapes: a volume is ``(..., nx, ny, nz)`` and a sinogram ``(..., n_angles,
n_h, n_v)`` (the library's internal layout, v fastest).  Leading batch
dimensions are projected together (``ccpi_forward_batch`` /
``ccpi_backward_batch``: one launch per direction for cone beam).
"""
from __future__ import annotations

import torch

from .device import Plan


def _batched(fwd, plan: Plan, src: torch.Tensor, in_shape, out_shape):
    if tuple(src.shape[-3:]) != tuple(in_shape):
        raise ValueError(f"expected trailing shape {tuple(in_shape)}, got {tuple(src.shape)}")
    lead = src.shape[:-3]
    flat = src.reshape((-1,) + tuple(in_shape))
    if not flat.is_contiguous():
        flat = flat.contiguous()
    out = torch.empty((flat.shape[0],) + tuple(out_shape), device=src.device, dtype=torch.float32)
    (plan.forward_batch if fwd else plan.backward_batch)(flat, out)
    return out.reshape(tuple(lead) + tuple(out_shape))


def forward_project(plan: Plan, vol: torch.Tensor) -> torch.Tensor:
    """A x for a volume or a batch of volumes (no autograd)."""
    return _batched(True, plan, vol, plan.shape, plan.sino_shape)


def back_project(plan: Plan, sino: torch.Tensor) -> torch.Tensor:
    """A^T y for a sinogram or a batch of sinograms (no autograd)."""
    return _batched(False, plan, sino, plan.sino_shape, plan.shape)


class ProjectFunction(torch.autograd.Function):
    """y = A x with dL/dx = A^T dL/dy."""

    @staticmethod
    def forward(ctx, vol, plan):
        if vol.dtype != torch.float32 or not vol.is_cuda:
            raise ValueError("volume must be a float32 CUDA tensor")
        ctx.plan = plan
        return forward_project(plan, vol.detach())

    @staticmethod
    def backward(ctx, grad_sino):
        g = grad_sino.detach()
        if g.dtype != torch.float32:
            g = g.float()
        return back_project(ctx.plan, g), None


class BackProjectFunction(torch.autograd.Function):
    """x = A^T y with dL/dy = A dL/dx."""

    @staticmethod
    def forward(ctx, sino, plan):
        if sino.dtype != torch.float32 or not sino.is_cuda:
            raise ValueError("sinogram must be a float32 CUDA tensor")
        ctx.plan = plan
        return back_project(plan, sino.detach())

    @staticmethod
    def backward(ctx, grad_vol):
        g = grad_vol.detach()
        if g.dtype != torch.float32:
            g = g.float()
        return forward_project(ctx.plan, g), None


def project(vol: torch.Tensor, plan: Plan) -> torch.Tensor:
    """Differentiable forward projection."""
    return ProjectFunction.apply(vol, plan)


def backproject(sino: torch.Tensor, plan: Plan) -> torch.Tensor:
    """Differentiable back projection."""
    return BackProjectFunction.apply(sino, plan)


class Projector(torch.nn.Module):
    """``torch.nn.Module`` holding one plan; ``forward(x) = A x``."""

    def __init__(self, plan: Plan):
        super().__init__()
        self.plan = plan

    def forward(self, vol):
        return project(vol, self.plan)

    def adjoint(self, sino):
        return backproject(sino, self.plan)
