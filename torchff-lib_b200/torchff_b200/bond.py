"""Harmonic bonds (interface of torchff/bond.py:9-110): E = 1/2 k (r - b0)^2 per bond.

``HarmonicBond`` keeps the reference constructor and ``forward`` signature; both paths of
``use_customized_ops`` run the sm_100a kernels of libtffb200 (there is no second
implementation). Bond lengths use no periodic image, as in the reference.
"""
from __future__ import annotations

import torch
import torch.nn as nn

from . import ops as _ops  # noqa: F401  (registers torch.ops.torchff.*)


@torch._dynamo.disable
def compute_harmonic_bond_energy(coords: torch.Tensor, bonds: torch.Tensor, b0: torch.Tensor,
                                 k: torch.Tensor) -> torch.Tensor:
    """Total harmonic bond energy (0-d); differentiable in coords, b0 and k."""
    return torch.ops.torchff.compute_harmonic_bond_energy(coords, bonds, b0, k)


def compute_harmonic_bond_forces(coords: torch.Tensor, bonds: torch.Tensor, b0: torch.Tensor, k: torch.Tensor,
                                 forces: torch.Tensor):
    """Adds the bond forces -dE/dx into ``forces`` in place (no autograd)."""
    return torch.ops.torchff.compute_harmonic_bond_forces(coords, bonds, b0, k, forces)


class HarmonicBond(nn.Module):
    def __init__(self, use_customized_ops: bool = False):
        super().__init__()
        self.use_customized_ops = use_customized_ops

    def forward(self, coords, bonds, b0, k):
        return compute_harmonic_bond_energy(coords, bonds, b0, k)
