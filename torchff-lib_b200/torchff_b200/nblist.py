"""Neighbour lists (interface of torchff/nblist.py:10-250).

``NeighborList`` keeps the reference constructor and ``forward`` signature. Both
algorithms run the sm_100a kernels of libtffb200: ``"nsquared"`` is a shared-memory
tiled all-pairs test, ``"cell_list"`` bins atoms on a Hilbert-ordered cell grid, groups
them in 32-atom clusters and tests cluster pairs with 32x32 warp tiles.
``use_customized_ops`` is accepted for signature compatibility; there is no second
implementation behind it.

When ``max_npairs`` is too small, the reference's ``NeighborList`` returns a truncated list
(torchff/nblist.py:162-178). Both kernels here count every pair past the capacity, so
``NeighborList`` builds once more with the exact size and returns the full list; pass
``grow_on_overflow=False`` to keep the truncation (with a warning).
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


# npairs of the cell list when a cluster's neighbour-cluster list overflowed (pair count unknown)
CLUSTER_LIST_OVERFLOW = 2 ** 31 - 1


class NeighborList(nn.Module):
    def __init__(self, natoms: int, exclusions: torch.Tensor | None = None, include_self: bool = False,
                 use_customized_ops: bool = True, algorithm: str = "nsquared", *, grow_on_overflow: bool = True):
        super().__init__()
        self.grow_on_overflow = grow_on_overflow
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
        if found == CLUSTER_LIST_OVERFLOW and self.algorithm == "cell_list":
            raise RuntimeError("cell list: a cluster has more neighbour clusters than the list holds "
                               "(cutoff too large for the cell grid); use algorithm='nsquared'")
        if found > pairs.shape[0]:
            if self.grow_on_overflow:
                # the count is exact: one more build with room for every pair
                return self.forward(coords, box, cutoff, found, padding)
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


def build_cluster_pairs(coords: torch.Tensor, box: torch.Tensor, cutoff: float,
                        exclusions: Optional[torch.Tensor] = None, cell_size: float = 0.4,
                        max_num_interacting_clusters: int = -1):
    """Cluster-pair neighbour format (torchff/nblist.py:260-285 signature).

    Returns ``(sorted_atom_indices, cluster_exclusions, bitmask_exclusions,
    interacting_clusters, interacting_atoms)``:

    - ``sorted_atom_indices`` int32 (nclusters*32,): atom at each slot of the Hilbert-ordered
      32-atom clusters, -1 after the last atom;
    - ``cluster_exclusions`` int32 (2, T): cluster pairs (x, y), x <= y, whose 32x32 tile holds
      an excluded pair, and every diagonal tile;
    - ``bitmask_exclusions`` uint32 (T, 32): bit j of row (t, i) set = pair (slot 32x+i,
      slot 32y+j) skipped (excluded, padding, or j <= i when x == y);
    - ``interacting_clusters`` int32 (M,), ``interacting_atoms`` int32 (M, 32): atoms of lower
      clusters within the cutoff of cluster x's bounding box, -1 padded.

    Every pair within the cutoff that is not excluded lies in exactly one tile or entry.
    ``exclusions`` is a (2, E) tensor of excluded atom pairs (either order). With
    ``max_num_interacting_clusters`` > 0 the entry arrays have that many rows (-1 padded)
    and a build that needs more raises; -1 sizes them exactly. ``cell_size`` is accepted
    for signature compatibility: the cell grid is chosen from the atom count.
    """
    return torch.ops.torchff.build_cluster_pairs(coords, box, cutoff, exclusions, cell_size,
                                                 max_num_interacting_clusters)


def decode_cluster_pairs(coords: torch.Tensor, box: torch.Tensor, sorted_atom_indices, cluster_exclusions,
                         bitmask_exclusions, interacting_clusters, interacting_atoms, cutoff: float,
                         max_npairs: int = -1, padding: bool = False) -> Tuple[torch.Tensor, torch.Tensor]:
    """Atom pairs of a cluster-pair format within the cutoff (torchff/nblist.py:288-311
    signature): int32 (P, 2) rows (larger, smaller) and npairs int32 (1,). ``max_npairs`` = -1
    sizes the output exactly; with ``padding`` the full (max_npairs, 2) buffer is returned,
    -1 after the found pairs."""
    return torch.ops.torchff.decode_cluster_pairs(coords, box, sorted_atom_indices, cluster_exclusions,
                                                  bitmask_exclusions, interacting_clusters, interacting_atoms,
                                                  cutoff, max_npairs, padding)


def build_neighbor_list_cluster_pairs(coords: torch.Tensor, box: torch.Tensor, cutoff: float,
                                      exclusions: Optional[torch.Tensor], cell_size: float = 0.45,
                                      max_num_interacting_clusters: int = -1, max_npairs: int = -1,
                                      padding: bool = False):
    """Pair list through the cluster-pair format (torchff/nblist.py:314-337)."""
    nblist = build_cluster_pairs(coords, box, cutoff, exclusions, cell_size, max_num_interacting_clusters)
    return decode_cluster_pairs(coords, box, *nblist, cutoff, max_npairs, padding)
