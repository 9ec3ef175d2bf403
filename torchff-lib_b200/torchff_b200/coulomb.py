"""Shifted-cutoff Coulomb over a pair list (interface of torchff/coulomb.py)."""
from __future__ import annotations

import torch
import torch.nn as nn

from . import ops as _ops  # noqa: F401


def compute_coulomb_energy(coords, pairs, box, charges, coulomb_constant: float, cutoff: float,
                           do_shift: bool = True) -> torch.Tensor:
    if pairs.dtype != torch.int64:
        pairs = pairs.to(torch.int64)
    return torch.ops.torchff.compute_coulomb_energy(coords, pairs, box, charges, coulomb_constant, cutoff, do_shift)


class Coulomb(nn.Module):
    def __init__(self, use_customized_ops: bool = False):
        super().__init__()
        self.use_customized_ops = use_customized_ops

    def forward(self, coords, pairs, box, charges, coulomb_constant: float, cutoff: float, do_shift: bool = True):
        return compute_coulomb_energy(coords, pairs, box, charges, coulomb_constant, cutoff, do_shift)
