"""The total energy as a torch.autograd.Function whose backward is the engine's adjoint.

``TotalEnergy.apply(engine, positions)`` takes positions of shape (natom, 3) in box units
(float64, any device) and returns the scalar U_total (kT) of the configuration, computed by
yamc_set_positions (the full recompute of mc_calc_total_sums).  The backward pass returns
-forces from yamc_forces, the hand-written adjoint of the same energy: real space with the
derivative of the piecewise erfc_Luc, k-space Coulomb and dispersion, and the external term.
Both directions run in libyamc_b200.so on the GPU; torch only carries the tensors.
"""
from __future__ import annotations

import numpy as np
import torch


class TotalEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, engine, positions: torch.Tensor) -> torch.Tensor:
        p = positions.detach().to("cpu", torch.float64).numpy()
        e = engine.set_positions(p[:, 0], p[:, 1], p[:, 2])
        f, _, _ = engine.forces()
        ctx.save_for_backward(torch.from_numpy(-f).to(positions.device))
        return torch.tensor(e[0], dtype=torch.float64, device=positions.device)

    @staticmethod
    def backward(ctx, grad_out):
        (grad,) = ctx.saved_tensors
        return None, grad_out * grad


def total_energy(engine, positions: torch.Tensor) -> torch.Tensor:
    return TotalEnergy.apply(engine, positions)
