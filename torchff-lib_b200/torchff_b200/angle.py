"""Angles and harmonic angle energies (interface of torchff/angle.py:8-200):
theta = angle at the central atom j of each (i, j, k); E = 1/2 k (theta - theta0)^2.

``Angles`` and ``HarmonicAngle`` keep the reference constructors and ``forward``
signatures; both paths of ``use_customized_ops`` run the sm_100a kernels of libtffb200.
"""
from __future__ import annotations

import torch
import torch.nn as nn

from . import ops as _ops  # noqa: F401  (registers torch.ops.torchff.*)


@torch._dynamo.disable
def compute_angles(coords: torch.Tensor, angles: torch.Tensor) -> torch.Tensor:
    """Angle (radians) of every (i, j, k) row of ``angles``; differentiable in coords."""
    return torch.ops.torchff.compute_angles(coords, angles)


class Angles(nn.Module):
    def __init__(self, use_customized_ops: bool = False):
        super().__init__()
        self.use_customized_ops = use_customized_ops

    def forward(self, coords: torch.Tensor, angles: torch.Tensor) -> torch.Tensor:
        return compute_angles(coords, angles)


@torch._dynamo.disable
def compute_harmonic_angle_energy(coords: torch.Tensor, angles: torch.Tensor, theta0: torch.Tensor,
                                  k: torch.Tensor) -> torch.Tensor:
    """Total harmonic angle energy (0-d); differentiable in coords, theta0 and k."""
    return torch.ops.torchff.compute_harmonic_angle_energy(coords, angles, theta0, k)


def compute_harmonic_angle_forces(coords: torch.Tensor, angles: torch.Tensor, theta0: torch.Tensor,
                                  k: torch.Tensor, forces: torch.Tensor) -> torch.Tensor:
    """Adds the angle forces -dE/dx into ``forces`` in place (no autograd); returns ``forces``."""
    torch.ops.torchff.compute_harmonic_angle_forces(coords, angles, theta0, k, forces)
    return forces


class HarmonicAngle(nn.Module):
    def __init__(self, use_customized_ops: bool = False):
        super().__init__()
        self.use_customized_ops = use_customized_ops

    def forward(self, coords, angles, theta0, k):
        return compute_harmonic_angle_energy(coords, angles, theta0, k)
