"""Neighbour lists (interface of torchff/nblist.py:10-250).

``NeighborList`` keeps the reference constructor and ``forward`` signature. Both
algorithms run the sm_100a kernels of libtffb200: ``"nsquared"`` is a shared-memory
tiled all-pairs test, ``"cell_list"`` bins atoms on a Morton-ordered cell grid, groups
them in 32-atom clusters and tests cluster pairs with 32x32 warp tiles.
``use_customized_ops`` is accepted for signature compatibility; there is no second
implementation behind it.
"""
from __future__ import annotations

import warnings
from typing import Optional, Tuple

import torch
import torch.nn as nn

from . import ops as _ops  # noqa: F401  (registers torch.ops.torchff.*)


def convert_pairs_coo_to_csr(pairs_coo: torch.Tensor, num_atoms: Optional[int] = None
                             ) -> Tuple[torch.Tensor, torch.Tensor]:
    """Symmetric CSR of an exclusion pair list (torchff/nblist.py:50-123 semantics).

    Both (i, j) and (j, i) end up in the structure, duplicates are removed, columns are
    sorted within each row.
    """
    both = torch.cat([pairs_coo, pairs_coo.flip(1)], dim=0).to(torch.long)
    if num_atoms is None:
        num_atoms = int(both.max().item()) + 1
    keys = torch.unique(both[:, 0] * num_atoms + both[:, 1])
    rows = keys // num_atoms
    cols = keys % num_atoms
    counts = torch.bincount(rows, minlength=num_atoms)
    row_ptr = torch.zeros(num_atoms + 1, dtype=torch.long, device=pairs_coo.device)
    row_ptr[1:] = torch.cumsum(counts, 0)
    return row_ptr, cols


class NeighborList(nn.Module):
    def __init__(self, natoms: int, exclusions: torch.Tensor | None = None, include_self: bool = False,
                 use_customized_ops: bool = True, algorithm: str = "nsquared"):
        super().__init__()
        if algorithm not in ("nsquared", "cell_list"):
            raise ValueError(f"algorithm must be 'nsquared' or 'cell_list', got '{algorithm}'")
        self.natoms = natoms
        self.include_self = include_self
        self.use_customized_ops = use_customized_ops
        self.algorithm = algorithm
        if exclusions is not None:
            self.register_buffer("exclusions_coo", exclusions.to(torch.long))
            rp, col = convert_pairs_coo_to_csr(exclusions, natoms)
            self.register_buffer("excl_row_ptr", rp)
            self.register_buffer("excl_col_indices", col)
        else:
            self.exclusions_coo = None
            self.excl_row_ptr = None
            self.excl_col_indices = None

    convert_pairs_coo_to_csr = staticmethod(convert_pairs_coo_to_csr)

    def to(self, *args, **kwargs):
        model = super().to(*args, **kwargs)
        for name in ("exclusions_coo", "excl_row_ptr", "excl_col_indices"):
            t = getattr(self, name, None)
            if t is not None:
                setattr(self, name, t.to(torch.long))
        return model

    def forward(self, coords: torch.Tensor, box: torch.Tensor, cutoff: float, max_npairs: int = -1,
                padding: bool = False):
        if self.algorithm == "cell_list":
            if box is None:
                raise ValueError("Cell-list algorithm requires a periodic box")
            pairs, npairs = torch.ops.torchff.build_neighbor_list_cell_list(
                coords, box, cutoff, max_npairs, self.excl_row_ptr, self.excl_col_indices, self.include_self)
        else:
            pairs, npairs = torch.ops.torchff.build_neighbor_list_nsquared(
                coords, box, cutoff, max_npairs, self.excl_row_ptr, self.excl_col_indices, self.include_self)
        if padding:
            return pairs, npairs
        found = int(npairs.item())
        if found > pairs.shape[0]:
            warnings.warn(f"neighbour list truncated: found {found} pairs, capacity {pairs.shape[0]}",
                          stacklevel=2)
        return pairs[:found]


def _trim(pairs, npairs, padding):
    if padding:
        return pairs, npairs
    found = int(npairs.item())
    if found > pairs.shape[0]:
        raise RuntimeError(f"Too many neighbor pairs found. Maximum is {pairs.shape[0]} but found {found}")
    return pairs[:found], npairs


def build_neighbor_list_nsquared(coords: torch.Tensor, box: torch.Tensor, cutoff: float, max_npairs: int = -1,
                                 padding: bool = False, excl_row_ptr: Optional[torch.Tensor] = None,
                                 excl_col_indices: Optional[torch.Tensor] = None, include_self: bool = False,
                                 out: Optional[torch.Tensor] = None):
    """Functional O(N^2) build (torchff/nblist.py:183-250)."""
    if out is not None:
        npairs = torch.ops.torchff.build_neighbor_list_nsquared_out(
            coords, box, cutoff, out, excl_row_ptr, excl_col_indices, include_self)
        return _trim(out, npairs, padding)
    pairs, npairs = torch.ops.torchff.build_neighbor_list_nsquared(
        coords, box, cutoff, max_npairs, excl_row_ptr, excl_col_indices, include_self)
    return _trim(pairs, npairs, padding)


def build_neighbor_list_cell_list(coords: torch.Tensor, box: torch.Tensor, cutoff: float, max_npairs: int = -1,
                                  padding: bool = False, excl_row_ptr: Optional[torch.Tensor] = None,
                                  excl_col_indices: Optional[torch.Tensor] = None, include_self: bool = False,
                                  out: Optional[torch.Tensor] = None):
    """Functional cluster/cell-list build with the output contract of the O(N^2) one."""
    if out is not None:
        _, npairs = torch.ops.torchff.build_neighbor_list_cell_list_out(
            coords, box, cutoff, out, excl_row_ptr, excl_col_indices, include_self)
        return _trim(out, npairs, padding)
    pairs, npairs = torch.ops.torchff.build_neighbor_list_cell_list(
        coords, box, cutoff, max_npairs, excl_row_ptr, excl_col_indices, include_self)
    return _trim(pairs, npairs, padding)
