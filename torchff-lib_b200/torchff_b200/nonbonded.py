"""Fused Coulomb + Lennard-Jones over a pair list (interface of torchff/nonbonded.py)."""
from __future__ import annotations

import torch
import torch.nn as nn

from . import ops as _ops  # noqa: F401


@torch._dynamo.disable
def compute_nonbonded_energy_from_atom_pairs(coords, pairs, box, sigma, epsilon, charges, coul_constant,
                                             cutoff: float, do_shift: bool = True) -> torch.Tensor:
    """E = sum_{r<=rc} k q_i q_j (1/r - [shift]/rc) + 4 eps_ij ((s_ij/r)^12 - (s_ij/r)^6), LB combining."""
    if pairs.dtype != torch.int64:
        pairs = pairs.to(torch.int64)
    return torch.ops.torchff.compute_nonbonded_energy_from_atom_pairs(
        coords, pairs, box, sigma, epsilon, charges, coul_constant, cutoff, do_shift)


def compute_nonbonded_forces_from_atom_pairs(coords, pairs, box, sigma, epsilon, charges, coul_constant,
                                             cutoff: float, forces: torch.Tensor) -> torch.Tensor:
    """Adds the shifted Coulomb + LJ forces into ``forces`` in place."""
    if pairs.dtype != torch.int64:
        pairs = pairs.to(torch.int64)
    torch.ops.torchff.compute_nonbonded_forces_from_atom_pairs(
        coords, pairs, box, sigma, epsilon, charges, coul_constant, cutoff, forces)
    return forces


def _k_tensor(coul_constant, like: torch.Tensor) -> torch.Tensor:
    if torch.is_tensor(coul_constant):
        return coul_constant
    return torch.tensor(float(coul_constant), dtype=like.dtype, device=like.device)


@torch._dynamo.disable
def compute_nonbonded_energy_from_cluster_pairs(coords, box, sigma, epsilon, charges, coul_constant,
                                                cutoff: float, sorted_atom_indices, cluster_exclusions,
                                                bitmask_exclusions, interacting_clusters, interacting_atoms,
                                                do_shift: bool = True) -> torch.Tensor:
    """The same energy as ``compute_nonbonded_energy_from_atom_pairs`` over the pairs of a
    cluster-pair format (``nblist.build_cluster_pairs``), without an int64 pair list.
    Differentiable in coords, sigma, epsilon, charges and a tensor ``coul_constant``."""
    return torch.ops.torchff.compute_nonbonded_energy_from_cluster_pairs(
        coords, box, sigma, epsilon, charges, _k_tensor(coul_constant, coords), cutoff, sorted_atom_indices,
        cluster_exclusions, bitmask_exclusions, interacting_clusters, interacting_atoms, do_shift)


def compute_nonbonded_forces_from_cluster_pairs(coords, box, sigma, epsilon, charges, coul_constant,
                                                cutoff: float, sorted_atom_indices, cluster_exclusions,
                                                bitmask_exclusions, interacting_clusters, interacting_atoms,
                                                forces: torch.Tensor) -> torch.Tensor:
    """Adds the shifted Coulomb + LJ forces over a cluster-pair format into ``forces``."""
    torch.ops.torchff.compute_nonbonded_forces_from_cluster_pairs(
        coords, box, sigma, epsilon, charges, _k_tensor(coul_constant, coords), cutoff, sorted_atom_indices,
        cluster_exclusions, bitmask_exclusions, interacting_clusters, interacting_atoms, forces)
    return forces


class Nonbonded(nn.Module):
    """Fused fixed-charge nonbonded (Coulomb + Lennard-Jones) interaction."""

    def __init__(self, use_customized_ops: bool = False):
        super().__init__()
        self.use_customized_ops = use_customized_ops

    def forward(self, coords, pairs, box, sigma, epsilon, charges, coul_constant: float, cutoff: float,
                do_shift: bool = True) -> torch.Tensor:
        return compute_nonbonded_energy_from_atom_pairs(coords, pairs, box, sigma, epsilon, charges, coul_constant,
                                                        cutoff, do_shift)
