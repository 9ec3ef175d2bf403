"""Real-space Ewald Coulomb for point charges (interface of torchff/multipoles.py:215-355, rank 0).

E = prefactor [sum_{pairs, r<=rc} q_i q_j erfc(a r)/r + sum_{excl, r<=rc} q_i q_j (erfc(a r) - 1)/r];
``ewald_alpha < 0`` selects plain 1/r Coulomb without the exclusion term. Ranks 1 and 2
(dipoles, quadrupoles) and ``return_fields`` are outside the fixed-charge path and raise.
"""
from __future__ import annotations

import torch
import torch.nn as nn

from . import ops as _ops  # noqa: F401


@torch._dynamo.disable
def compute_multipolar_energy_from_atom_pairs(coords, box, pairs, pairs_excl, q, p, t, cutoff: float,
                                              ewald_alpha: float, prefactor: float) -> torch.Tensor:
    return torch.ops.torchff.compute_multipolar_energy_from_atom_pairs(
        coords, box, pairs, pairs_excl, q, p, t, cutoff, ewald_alpha, prefactor)


class MultipolarInteraction(nn.Module):
    def __init__(self, rank: int, cutoff: float, ewald_alpha: float = -1.0, prefactor: float = 1.0,
                 return_fields: bool = False, use_customized_ops: bool = True, cuda_graph_compat: bool = True):
        super().__init__()
        if rank != 0:
            raise NotImplementedError("only rank 0 (point charges) is implemented")
        if return_fields:
            raise NotImplementedError("return_fields is not implemented")
        self.rank = rank
        self.cutoff = cutoff
        self.ewald_alpha = ewald_alpha
        self.prefactor = prefactor
        self.return_fields = return_fields
        self.use_customized_ops = use_customized_ops
        self.cuda_graph_compat = cuda_graph_compat

    def forward(self, coords, box, pairs, q, p=None, t=None, pairs_excl=None):
        if pairs.dtype != torch.int64:
            pairs = pairs.to(torch.int64)
        return compute_multipolar_energy_from_atom_pairs(coords, box, pairs, pairs_excl, q, p, t, self.cutoff,
                                                         self.ewald_alpha, self.prefactor)
