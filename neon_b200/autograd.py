"""torch.autograd harness over the device adjoint.

``equilibrium_displacement(G, problem)`` returns the equilibrium displacement u(G) of a
microsphere problem for a per-element shear-modulus field G (a torch tensor); its backward pass
is the hand-written adjoint (nb2_adjoint_shear_gradient): one transpose solve on the converged
tangent plus the element kernel for df_int/dG.  The forward solve is neon's static_matrix
(nb2_static_solve).  Tensors cross the boundary on the host (the C-ABI takes host buffers).
"""
from __future__ import annotations

import copy

import numpy as np
import torch

from . import api


class _Equilibrium(torch.autograd.Function):
    @staticmethod
    def forward(ctx, G, problem, precision, tolerance):
        pr = copy.copy(problem)
        pr.element_shear_modulus = G.detach().cpu().numpy().astype(np.float64)
        sm = api.StaticMatrix(pr, precision=precision)
        u = sm.solve()
        ctx.sm = sm
        ctx.precision = precision
        ctx.tolerance = tolerance
        return torch.from_numpy(u).to(G.device)

    @staticmethod
    def backward(ctx, grad_u):
        g = ctx.sm.mesh.adjoint_shear_gradient(grad_u.detach().cpu().numpy(), ctx.precision,
                                               ctx.tolerance)
        ctx.sm.mesh.close()
        return torch.from_numpy(g).to(grad_u.device), None, None, None


def equilibrium_displacement(G: torch.Tensor, problem, precision=api.FP64,
                             tolerance: float = 1e-12) -> torch.Tensor:
    """u(G) with d u / d G available through the adjoint (float64 tensors)."""
    return _Equilibrium.apply(G, problem, precision, tolerance)
