"""torch.autograd.Function over the adjoint-gradient kernels.

``ExpectationFunction.apply(theta, n, ops, observable)`` returns
E_b = <psi(theta_b)|H|psi(theta_b)> (float64, shape [B]) for a batch of
parameter vectors theta [B, P]; backward multiplies the FP64 adjoint
gradients (computed in the same libqsim call as E) by grad_output.  The
reference has no differentiation (ROADMAP.md:173-175).
"""
from __future__ import annotations

import numpy as np
import torch

from . import engine as E


class ExpectationFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta, n_qubits, ops, observable):
        th = theta.detach().to("cpu", torch.float64)
        squeeze = th.dim() == 1
        th2 = th.reshape(1, -1) if squeeze else th
        energies, grads = E.adjoint_gradient(int(n_qubits), ops, th2.shape[1], th2.numpy(), observable)
        g = torch.from_numpy(grads).to(theta.device, theta.dtype)
        ctx.save_for_backward(g.reshape(theta.shape))
        out = torch.from_numpy(energies).to(theta.device, theta.dtype)
        return out.reshape(()) if squeeze else out

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        if g.dim() == 1:
            return grad_out * g, None, None, None
        return grad_out.reshape(-1, 1) * g, None, None, None


def expectation(theta: torch.Tensor, n_qubits: int, ops: np.ndarray, observable) -> torch.Tensor:
    return ExpectationFunction.apply(theta, n_qubits, ops, observable)
