"""torch.ops.torchff.* on libtffb200: the reference's operator schemas, re-registered.

The reference's registered operators (csrc/nblist/nblist_interface.cpp:4-9,
csrc/nonbonded/nonbonded_interface.cpp:4-11, csrc/coulomb/coulomb_interface.cpp:5-7,
csrc/vdw/vdw_interface.cpp:5-8, csrc/multipoles/multipoles_interface.cpp:5-9,
csrc/pme/pme_interface.cpp:5-14, csrc/bond/bond_interface.cpp:5-6,
csrc/angle/angle_interface.cpp:5-8) are registered in C++ by libtffb200_torch.so
(csrc/torch_ops.cpp), which this module loads: Python callers, TorchScript modules and C++
hosts without Python reach the same kernels. Neighbour lists run on ``CUDA``, energy terms
on ``AutogradCUDA`` (plus ``CUDA`` for autograd-free calls); each energy op computes the
energy and every requested first derivative in one forward launch and backward scales
them by the incoming gradient (csrc/nonbonded/nonbonded_atom_pairs_cuda.cu:220-237).

This module adds the cluster-pair format, which the reference has as Python entry points
(torchff/nblist.py:260-311) and kernels but no registered schema.

Only rank-0 (point charge) multipolar/PME calls and Lennard-Jones vdW are implemented;
other ranks and the buffered 14-7 potential raise NotImplementedError.
"""
from __future__ import annotations

import os

import torch

from . import _lib as L
from ._build import torch_lib_path


def _load_operator_library() -> None:
    p = torch_lib_path()
    if not os.path.exists(p):
        raise ImportError(f"{p} is missing: build it with torchff-lib_b200/torchff_b200/_build.py")
    torch.ops.load_library(p)


_load_operator_library()

_DEF = torch.library.Library("torchff", "FRAGMENT")

# cluster-pair format: the reference has these Python entry points (torchff/nblist.py:260-311) and
# kernels (csrc/nblist/nblist_cluster_pairs_cuda.cu, csrc/nonbonded/nonbonded_cluster_pairs_cuda.cu)
# but no registered schema; the energy/forces schemas follow its commented-out definitions
# (csrc/nonbonded/nonbonded_interface.cpp:7-8)
SCHEMAS = {
    "build_cluster_pairs": "build_cluster_pairs(Tensor coords, Tensor box, Scalar cutoff, Tensor? exclusions, Scalar cell_size, Scalar max_num_interacting_clusters) -> (Tensor, Tensor, Tensor, Tensor, Tensor)",
    "decode_cluster_pairs": "decode_cluster_pairs(Tensor coords, Tensor box, Tensor sorted_atom_indices, Tensor cluster_exclusions, Tensor bitmask_exclusions, Tensor interacting_clusters, Tensor interacting_atoms, Scalar cutoff, Scalar max_npairs, bool padding) -> (Tensor, Tensor)",
    "compute_nonbonded_energy_from_cluster_pairs": "compute_nonbonded_energy_from_cluster_pairs(Tensor coords, Tensor box, Tensor sigma, Tensor epsilon, Tensor charges, Tensor coul_constant, Scalar cutoff, Tensor sorted_atom_indices, Tensor cluster_exclusions, Tensor bitmask_exclusions, Tensor interacting_clusters, Tensor interacting_atoms, bool do_shift) -> Tensor",
    "compute_nonbonded_forces_from_cluster_pairs": "compute_nonbonded_forces_from_cluster_pairs(Tensor coords, Tensor box, Tensor sigma, Tensor epsilon, Tensor charges, Tensor coul_constant, Scalar cutoff, Tensor sorted_atom_indices, Tensor cluster_exclusions, Tensor bitmask_exclusions, Tensor interacting_clusters, Tensor interacting_atoms, Tensor forces) -> ()",
}
for _s in SCHEMAS.values():
    _DEF.define(_s)


def _c(t: torch.Tensor | None, dtype=None) -> torch.Tensor | None:
    if t is None:
        return None
    if dtype is not None and t.dtype != dtype:
        t = t.to(dtype)
    return t.contiguous()


def _long(t: torch.Tensor | None) -> torch.Tensor | None:
    return _c(t, torch.int64)


# ---------------------------------------------------------------------------------------
# cluster-pair format (dispatch key CUDA for build / decode, AutogradCUDA for the energy)
# ---------------------------------------------------------------------------------------

# Initial capacity of interacting entries per cluster when the caller gives none; a build
# that needs more runs once more with the exact count (water at rc = 1 nm needs ~30).
_ENTRIES_PER_CLUSTER = 64


def _build_cluster_pairs(coords, box, cutoff, exclusions, cell_size, max_num_interacting_clusters):
    """The format of tff_cluster_pairs_build. ``cell_size`` is accepted for signature
    compatibility: the cell grid is chosen from the atom count (about 8 atoms per cell)."""
    from .nblist import convert_pairs_coo_to_csr

    L.require_cuda(coords, box, exclusions)
    x = _c(coords.detach())
    dt = x.dtype
    b = _c(box.detach(), dt)
    n = x.shape[0]
    dev = x.device
    rp = col = None
    if exclusions is not None and exclusions.numel() > 0:
        e = exclusions.detach().to(torch.long)
        if e.dim() != 2 or e.shape[0] != 2:
            raise RuntimeError("exclusions must be a (2, E) tensor of excluded atom pairs")
        if int(e.min()) < 0 or int(e.max()) >= n:
            raise RuntimeError(f"exclusions must index atoms in [0, {n})")
        rp, col = convert_pairs_coo_to_csr(e.t(), n)
    ncl = (n + 31) // 32
    user_cap = int(max_num_interacting_clusters)
    cap_t = ncl + (int(col.numel()) if col is not None else 0)
    cap_e = user_cap if user_cap > 0 else ncl * _ENTRIES_PER_CLUSTER
    dtc = L.dtype_code(dt)
    ws = L.workspace(L.lib.tff_cluster_pairs_workspace_bytes(dtc, n, 0), dev)
    counts = torch.zeros(3, dtype=torch.int64, device=dev)
    sorted_atoms = torch.empty(ncl * 32, dtype=torch.int32, device=dev)
    tiles = torch.empty((2, cap_t), dtype=torch.int32, device=dev)
    masks = torch.empty((cap_t, 32), dtype=torch.uint32, device=dev)
    while True:  # at most twice: a second build with the exact entry count
        ecl = torch.empty(cap_e, dtype=torch.int32, device=dev)
        eat = torch.empty((cap_e, 32), dtype=torch.int32, device=dev)
        L.check(L.lib.tff_cluster_pairs_build(dtc, n, L.ptr(x), L.ptr(b), float(cutoff), L.ptr(rp), L.ptr(col),
                                              L.ptr(sorted_atoms), L.ptr(tiles), L.ptr(masks), cap_t, L.ptr(ecl),
                                              L.ptr(eat), cap_e, L.ptr(counts), 0, L.ptr(ws), ws.numel(),
                                              L.stream_of(x)), "build_cluster_pairs")
        nt, ne, status = (int(v) for v in counts.tolist())
        if status & 1:
            raise RuntimeError("build_cluster_pairs: a 32-atom cluster has excluded partners in more than 64 clusters")
        if status & 2:
            raise RuntimeError("build_cluster_pairs: a cluster has more than 1024 neighbour clusters (cutoff too large)")
        if ne <= cap_e:
            break
        if user_cap > 0:
            raise RuntimeError(f"build_cluster_pairs: {ne} interacting entries needed, "
                               f"max_num_interacting_clusters is {user_cap}")
        cap_e = ne
    tiles = tiles[:, :nt].contiguous()
    masks = masks[:nt]
    if user_cap <= 0:
        ecl, eat = ecl[:ne], eat[:ne]
    return sorted_atoms, tiles, masks, ecl, eat


def _format_views(sorted_atom_indices, cluster_exclusions, bitmask_exclusions, interacting_clusters,
                  interacting_atoms):
    sa = _c(sorted_atom_indices.detach(), torch.int32)
    tiles = cluster_exclusions.detach()
    if tiles.dim() != 2 or tiles.shape[0] != 2:
        raise RuntimeError("cluster_exclusions must be a (2, T) tensor")
    tiles = _c(tiles, torch.int32)
    masks = bitmask_exclusions.detach()
    if masks.element_size() != 4 or masks.shape[0] != tiles.shape[1]:
        raise RuntimeError("bitmask_exclusions must be a (T, 32) tensor of 32-bit words")
    masks = masks.contiguous()
    ecl = _c(interacting_clusters.detach(), torch.int32)
    eat = _c(interacting_atoms.detach(), torch.int32)
    if eat.shape[0] != ecl.shape[0]:
        raise RuntimeError("interacting_atoms must have one row of 32 atoms per interacting cluster")
    return sa, tiles, masks, ecl, eat


def _decode_cluster_pairs(coords, box, sorted_atom_indices, cluster_exclusions, bitmask_exclusions,
                          interacting_clusters, interacting_atoms, cutoff, max_npairs, padding):
    """Pairs (larger, smaller) int32 of the format within the cutoff. max_npairs = -1 sizes the
    output exactly (a counting pass first) instead of N(N-1)/2 rows."""
    L.require_cuda(coords, box, sorted_atom_indices, cluster_exclusions, bitmask_exclusions, interacting_clusters,
                   interacting_atoms)
    x = _c(coords.detach())
    b = _c(box.detach(), x.dtype)
    sa, tiles, masks, ecl, eat = _format_views(sorted_atom_indices, cluster_exclusions, bitmask_exclusions,
                                               interacting_clusters, interacting_atoms)
    npairs = torch.zeros(1, dtype=torch.int32, device=x.device)

    def run(pairs, cap):
        L.check(L.lib.tff_cluster_pairs_decode(L.dtype_code(x.dtype), x.shape[0], L.ptr(x), L.ptr(b), float(cutoff),
                                               L.ptr(sa), sa.numel(), L.ptr(tiles), tiles.shape[1], L.ptr(masks),
                                               L.ptr(ecl), L.ptr(eat), ecl.shape[0], L.ptr(pairs), cap,
                                               L.ptr(npairs), L.stream_of(x)), "decode_cluster_pairs")

    cap = int(max_npairs)
    if cap < 0:
        run(None, 0)
        cap = int(npairs.item())
    pairs = torch.empty((cap, 2), dtype=torch.int32, device=x.device)
    run(pairs, cap)
    if padding:
        return pairs, npairs
    found = int(npairs.item())
    if found > cap:
        raise RuntimeError(f"Too many neighbor pairs found. Maximum is {cap} but found {found}")
    return pairs[:found], npairs


_DEF.impl("build_cluster_pairs", _build_cluster_pairs, "CUDA")
_DEF.impl("decode_cluster_pairs", _decode_cluster_pairs, "CUDA")


# ---------------------------------------------------------------------------------------
# nonbonded energy over the cluster-pair format
# ---------------------------------------------------------------------------------------

def _empty_like_or_none(t, want):
    return torch.empty_like(t) if want else None


def nonbonded_cluster_forward(coords, box, sigma, epsilon, charges, coul_constant, cutoff, sorted_atom_indices,
                              cluster_exclusions, bitmask_exclusions, interacting_clusters, interacting_atoms,
                              do_shift, need=(False, False, False, False, False)):
    """Energy (1,) over the cluster-pair format and optional dE/dx, dE/dsigma, dE/depsilon,
    dE/dq, dE/dk (``need`` in that order)."""
    L.require_cuda(coords, box, sigma, epsilon, charges, sorted_atom_indices, cluster_exclusions,
                   bitmask_exclusions, interacting_clusters, interacting_atoms)
    x = _c(coords.detach())
    dt = x.dtype
    b, s, e, q = (_c(t.detach(), dt) for t in (box, sigma, epsilon, charges))
    k = float(coul_constant.detach().reshape(-1)[0]) if torch.is_tensor(coul_constant) else float(coul_constant)
    sa, tiles, masks, ecl, eat = _format_views(sorted_atom_indices, cluster_exclusions, bitmask_exclusions,
                                               interacting_clusters, interacting_atoms)
    ene = torch.empty(1, dtype=dt, device=x.device)
    ecoul = torch.empty(1, dtype=dt, device=x.device) if need[4] else None
    gx = _empty_like_or_none(x, need[0])
    gs = _empty_like_or_none(s, need[1])
    ge = _empty_like_or_none(e, need[2])
    gq = _empty_like_or_none(q, need[3])
    dtc = L.dtype_code(dt)
    ws = L.workspace(L.lib.tff_nonbonded_cluster_pairs_workspace_bytes(dtc, x.shape[0]), x.device)

    def run(kc, energy, energy_c, gx_, gs_, ge_, gq_):
        L.check(L.lib.tff_nonbonded_cluster_pairs(dtc, x.shape[0], L.ptr(x), L.ptr(b), L.ptr(s), L.ptr(e), L.ptr(q),
                                                  kc, float(cutoff), int(bool(do_shift)), L.ptr(sa), sa.numel(),
                                                  L.ptr(tiles), tiles.shape[1], L.ptr(masks), L.ptr(ecl),
                                                  L.ptr(eat), ecl.shape[0], L.ptr(energy), L.ptr(energy_c),
                                                  L.ptr(gx_), L.ptr(gs_), L.ptr(ge_), L.ptr(gq_), L.ptr(ws),
                                                  ws.numel(), L.stream_of(x)),
                "compute_nonbonded_energy_from_cluster_pairs")

    run(k, ene, ecoul if k != 0.0 else None, gx, gs, ge, gq)
    gk = None
    if need[4]:
        if k != 0.0:
            gk = ecoul / k
        else:  # the Coulomb sum per unit k
            run(1.0, None, ecoul, None, None, None, None)
            gk = ecoul
    return ene, gx, gs, ge, gq, gk


class _NonbondedClusterFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coords, box, sigma, epsilon, charges, coul_constant, cutoff, sa, tiles, masks, ecl, eat,
                do_shift):
        ni = ctx.needs_input_grad
        ene, gx, gs, ge, gq, gk = nonbonded_cluster_forward(coords, box, sigma, epsilon, charges, coul_constant,
                                                            cutoff, sa, tiles, masks, ecl, eat, do_shift,
                                                            (ni[0], ni[2], ni[3], ni[4], ni[5]))
        ctx.k_shape = coul_constant.shape if torch.is_tensor(coul_constant) else None
        ctx.save_for_backward(gx, gs, ge, gq, gk)
        return ene

    @staticmethod
    def backward(ctx, g):
        gx, gs, ge, gq, gk = ctx.saved_tensors
        sc = lambda t: None if t is None else t * g
        gk_out = None
        if gk is not None and ctx.k_shape is not None:
            gk_out = (gk * g).reshape(ctx.k_shape) if len(ctx.k_shape) else (gk * g).reshape(())
        return sc(gx), None, sc(gs), sc(ge), sc(gq), gk_out, None, None, None, None, None, None, None


def _nonbonded_cluster_autograd(*args):
    return _NonbondedClusterFn.apply(*args)


def _nonbonded_cluster_cuda(*args):
    return nonbonded_cluster_forward(*args)[0]


def _nonbonded_cluster_forces(coords, box, sigma, epsilon, charges, coul_constant, cutoff, sorted_atom_indices,
                              cluster_exclusions, bitmask_exclusions, interacting_clusters, interacting_atoms,
                              forces):
    L.require_cuda(coords, box, sigma, epsilon, charges, forces)
    x = _c(coords.detach())
    dt = x.dtype
    if forces.dtype != dt or not forces.is_contiguous() or forces.shape != x.shape:
        raise RuntimeError("forces must be a contiguous tensor shaped and typed like coords")
    b, s, e, q = (_c(t.detach(), dt) for t in (box, sigma, epsilon, charges))
    k = float(coul_constant.detach().reshape(-1)[0]) if torch.is_tensor(coul_constant) else float(coul_constant)
    sa, tiles, masks, ecl, eat = _format_views(sorted_atom_indices, cluster_exclusions, bitmask_exclusions,
                                               interacting_clusters, interacting_atoms)
    dtc = L.dtype_code(dt)
    ws = L.workspace(L.lib.tff_nonbonded_cluster_pairs_workspace_bytes(dtc, x.shape[0]), x.device)
    L.check(L.lib.tff_nonbonded_forces_cluster_pairs(dtc, x.shape[0], L.ptr(x), L.ptr(b), L.ptr(s), L.ptr(e),
                                                     L.ptr(q), k, float(cutoff), L.ptr(sa), sa.numel(), L.ptr(tiles),
                                                     tiles.shape[1], L.ptr(masks), L.ptr(ecl), L.ptr(eat),
                                                     ecl.shape[0], L.ptr(forces), L.ptr(ws), ws.numel(),
                                                     L.stream_of(x)),
            "compute_nonbonded_forces_from_cluster_pairs")


_DEF.impl("compute_nonbonded_energy_from_cluster_pairs", _nonbonded_cluster_autograd, "AutogradCUDA")
_DEF.impl("compute_nonbonded_energy_from_cluster_pairs", _nonbonded_cluster_cuda, "CUDA")
_DEF.impl("compute_nonbonded_forces_from_cluster_pairs", _nonbonded_cluster_forces, "CUDA")
