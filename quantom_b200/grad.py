"""torch.autograd bridge to the engine's trajectory-loss adjoint.

``trajectory_loss(theta, engine, **spec)`` returns the loss of lima_loss /
lima_grad (include/lima_abi.h) as a 0-d tensor of theta's dtype; its
backward is d loss / d theta from the hand-written adjoint of the unrolled
steps (lima_grad), so the engine's force-field parameters can sit inside a
PyTorch optimisation loop.  theta follows Engine.get_params(): per-type sigma,
per-type epsilon, then the bond / angle / dihedral force-constant scales.
"""
from __future__ import annotations

import torch


class TrajectoryLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta, engine, spec):
        engine.set_params(theta.detach().to("cpu", torch.float64).numpy())
        if theta.requires_grad:
            loss, g = engine.grad(**spec)
            ctx.save_for_backward(torch.from_numpy(g).to(theta))
        else:
            loss = engine.loss(**spec)
        return theta.new_tensor(loss)

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        return grad_out * g, None, None


def trajectory_loss(theta: torch.Tensor, engine, **spec) -> torch.Tensor:
    """spec: n_steps, checkpoint_every, n_bins, r_max, w_energy, w_rdf, target."""
    return TrajectoryLoss.apply(theta, engine, spec)
