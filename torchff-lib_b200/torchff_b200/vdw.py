"""Lennard-Jones 12-6 over a pair list (interface of torchff/vdw.py).

Per-pair sigma/epsilon of shape (P,) or type tables (T, T) indexed through ``atom_types``.
The AMOEBA buffered 14-7 form is outside the fixed-charge path and raises.
"""
from __future__ import annotations

from typing import Literal, Optional

import torch
import torch.nn as nn

from . import ops as _ops  # noqa: F401


@torch._dynamo.disable
def compute_lennard_jones_energy(coords, pairs, box, sigma, epsilon, cutoff: float,
                                 atom_types: torch.Tensor | None = None) -> torch.Tensor:
    if pairs.dtype != torch.int64:
        pairs = pairs.to(torch.int64)
    return torch.ops.torchff.compute_lennard_jones_energy(coords, pairs, box, sigma, epsilon, cutoff, atom_types)


@torch._dynamo.disable
def compute_vdw_14_7_energy(coords, pairs, box, sigma, epsilon, cutoff: float,
                            atom_types: torch.Tensor | None = None) -> torch.Tensor:
    return torch.ops.torchff.compute_vdw_14_7_energy(coords, pairs, box, sigma, epsilon, cutoff, atom_types)


class Vdw(nn.Module):
    def __init__(self, function: Literal["LennardJones", "AmoebaVdw147"] = "LennardJones",
                 cutoff: Optional[float] = None, use_customized_ops: bool = False, use_type_pairs: bool = False,
                 sum_output: bool = True, cuda_graph_compat: bool = True):
        super().__init__()
        if function not in ("LennardJones", "AmoebaVdw147"):
            raise AssertionError(f"Invalid vdw function: {function}")
        if not sum_output:
            raise ValueError("sum_output must be True: the kernels return the total energy only")
        self.function = function
        self.cutoff = cutoff
        self.use_customized_ops = use_customized_ops
        self.use_type_pairs = use_type_pairs
        self.sum_output = sum_output
        self.cuda_graph_compat = cuda_graph_compat

    def forward(self, coords, pairs, box, sigma, epsilon, cutoff: float, atom_types: torch.Tensor | None = None):
        types = atom_types if self.use_type_pairs else None
        if self.function == "LennardJones":
            return compute_lennard_jones_energy(coords, pairs, box, sigma, epsilon, cutoff, types)
        return compute_vdw_14_7_energy(coords, pairs, box, sigma, epsilon, cutoff, types)
