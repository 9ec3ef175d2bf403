"""torch.ops.torchff.* on libtffb200: the reference's operator schemas, re-registered.

Schemas are those of the reference (csrc/nblist/nblist_interface.cpp:4-9,
csrc/nonbonded/nonbonded_interface.cpp:4-11, csrc/coulomb/coulomb_interface.cpp:5-7,
csrc/vdw/vdw_interface.cpp:5-8, csrc/multipoles/multipoles_interface.cpp:5-9,
csrc/pme/pme_interface.cpp:5-14) with the same dispatch keys: neighbour lists on
``CUDA``, energy terms on ``AutogradCUDA`` (plus ``CUDA`` for autograd-free calls).

As in the reference, each energy op computes the energy and every requested first
derivative in one forward launch; backward scales the saved derivatives by the incoming
gradient (csrc/nonbonded/nonbonded_atom_pairs_cuda.cu:220-237). Output shapes follow the
reference: (1,) for the nonbonded and Coulomb ops, 0-d for LJ, multipolar and PME.

Only rank-0 (point charge) multipolar/PME calls and Lennard-Jones vdW are implemented;
other ranks and the buffered 14-7 potential raise NotImplementedError.
"""
from __future__ import annotations

import threading

import torch

from . import _lib as L

_DEF = torch.library.Library("torchff", "DEF")

SCHEMAS = {
    "build_neighbor_list_nsquared": "build_neighbor_list_nsquared(Tensor coords, Tensor? box, Scalar cutoff, Scalar max_npairs, Tensor? excl_row_ptr, Tensor? excl_col_indices, bool include_self) -> (Tensor, Tensor)",
    "build_neighbor_list_nsquared_out": "build_neighbor_list_nsquared_out(Tensor coords, Tensor? box, Scalar cutoff, Tensor(a!) pairs, Tensor? excl_row_ptr, Tensor? excl_col_indices, bool include_self) -> Tensor",
    "build_neighbor_list_cell_list": "build_neighbor_list_cell_list(Tensor coords, Tensor? box, Scalar cutoff, Scalar max_npairs, Tensor? excl_row_ptr, Tensor? excl_col_indices, bool include_self) -> (Tensor, Tensor)",
    "build_neighbor_list_cell_list_out": "build_neighbor_list_cell_list_out(Tensor coords, Tensor? box, Scalar cutoff, Tensor(a!) pairs, Tensor? excl_row_ptr, Tensor? excl_col_indices, bool include_self) -> (Tensor, Tensor)",
    "compute_nonbonded_energy_from_atom_pairs": "compute_nonbonded_energy_from_atom_pairs(Tensor coords, Tensor pairs, Tensor box, Tensor sigma, Tensor epsilon, Tensor charges, Scalar coul_constant, Scalar cutoff, bool do_shift) -> Tensor",
    "compute_nonbonded_forces_from_atom_pairs": "compute_nonbonded_forces_from_atom_pairs(Tensor coords, Tensor pairs, Tensor box, Tensor sigma, Tensor epsilon, Tensor charges, Scalar coul_constant, Scalar cutoff, Tensor forces) -> ()",
    "compute_coulomb_energy": "compute_coulomb_energy(Tensor coords, Tensor pairs, Tensor box, Tensor charges, Scalar coulomb_constant, Scalar cutoff, bool do_shift) -> Tensor",
    "compute_lennard_jones_energy": "compute_lennard_jones_energy(Tensor coords, Tensor pairs, Tensor box, Tensor sigma, Tensor epsilon, Scalar cutoff, Tensor? atom_types) -> Tensor",
    "compute_vdw_14_7_energy": "compute_vdw_14_7_energy(Tensor coords, Tensor pairs, Tensor box, Tensor radius, Tensor epsilon, Scalar cutoff, Tensor? atom_types) -> Tensor",
    "compute_multipolar_energy_from_atom_pairs": "compute_multipolar_energy_from_atom_pairs(Tensor coords, Tensor box, Tensor pairs, Tensor? pairs_excl, Tensor q, Tensor? p, Tensor? t, Scalar cutoff, Scalar ewald_alpha, Scalar prefactor) -> Tensor",
    # cluster-pair format: the reference has these Python entry points (torchff/nblist.py:260-311) and
    # kernels (csrc/nblist/nblist_cluster_pairs_cuda.cu, csrc/nonbonded/nonbonded_cluster_pairs_cuda.cu)
    # but no registered schema; the energy/forces schemas follow its commented-out definitions
    # (csrc/nonbonded/nonbonded_interface.cpp:7-8)
    "build_cluster_pairs": "build_cluster_pairs(Tensor coords, Tensor box, Scalar cutoff, Tensor? exclusions, Scalar cell_size, Scalar max_num_interacting_clusters) -> (Tensor, Tensor, Tensor, Tensor, Tensor)",
    "decode_cluster_pairs": "decode_cluster_pairs(Tensor coords, Tensor box, Tensor sorted_atom_indices, Tensor cluster_exclusions, Tensor bitmask_exclusions, Tensor interacting_clusters, Tensor interacting_atoms, Scalar cutoff, Scalar max_npairs, bool padding) -> (Tensor, Tensor)",
    "compute_nonbonded_energy_from_cluster_pairs": "compute_nonbonded_energy_from_cluster_pairs(Tensor coords, Tensor box, Tensor sigma, Tensor epsilon, Tensor charges, Tensor coul_constant, Scalar cutoff, Tensor sorted_atom_indices, Tensor cluster_exclusions, Tensor bitmask_exclusions, Tensor interacting_clusters, Tensor interacting_atoms, bool do_shift) -> Tensor",
    "compute_nonbonded_forces_from_cluster_pairs": "compute_nonbonded_forces_from_cluster_pairs(Tensor coords, Tensor box, Tensor sigma, Tensor epsilon, Tensor charges, Tensor coul_constant, Scalar cutoff, Tensor sorted_atom_indices, Tensor cluster_exclusions, Tensor bitmask_exclusions, Tensor interacting_clusters, Tensor interacting_atoms, Tensor forces) -> ()",
    # bonded terms (csrc/bond/bond_interface.cpp:5-6, csrc/angle/angle_interface.cpp:5-8)
    "compute_harmonic_bond_energy": "compute_harmonic_bond_energy(Tensor coords, Tensor pairs, Tensor b0, Tensor k) -> Tensor",
    "compute_harmonic_bond_forces": "compute_harmonic_bond_forces(Tensor coords, Tensor pairs, Tensor b0, Tensor k, Tensor(a!) forces) -> ()",
    "compute_harmonic_angle_energy": "compute_harmonic_angle_energy(Tensor coords, Tensor angles, Tensor theta0, Tensor k) -> Tensor",
    "compute_harmonic_angle_forces": "compute_harmonic_angle_forces(Tensor coords, Tensor angles, Tensor theta0, Tensor k, Tensor(a!) forces) -> ()",
    "compute_angles": "compute_angles(Tensor coords, Tensor angles) -> Tensor",
    "pme_long_range": "pme_long_range(Tensor coords, Tensor box, Tensor q, Tensor? p, Tensor? t, Scalar K, Scalar alpha, Tensor xmoduli, Tensor ymoduli, Tensor zmoduli) -> Tensor",
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
# neighbour lists (dispatch key CUDA, no autograd: csrc/nblist/nblist_nsquared_cuda.cu:201)
# ---------------------------------------------------------------------------------------

def _nblist_out(algorithm: str, coords, box, cutoff, pairs, rp, col, include_self):
    L.require_cuda(coords, box, pairs, rp, col)
    x = _c(coords.detach())
    if pairs.dtype != torch.int64 or not pairs.is_contiguous() or pairs.dim() != 2 or pairs.shape[1] != 2:
        raise RuntimeError("pairs must be a contiguous (max_npairs, 2) int64 tensor")
    b = _c(box.detach(), x.dtype) if box is not None else None
    rp, col = _long(rp), _long(col)
    n = x.shape[0]
    npairs = torch.zeros(1, dtype=torch.int32, device=x.device)
    dt = L.dtype_code(x.dtype)
    stream = L.stream_of(x)
    if algorithm == "nsquared":
        L.check(L.lib.tff_nblist_nsquared(dt, n, L.ptr(x), L.ptr(b), float(cutoff), L.ptr(rp), L.ptr(col),
                                          int(bool(include_self)), L.ptr(pairs), pairs.shape[0], L.ptr(npairs),
                                          stream), "build_neighbor_list_nsquared")
    else:
        if b is None:
            raise RuntimeError("Cell-list neighbor list requires a periodic box")
        wsb = L.lib.tff_nblist_cell_list_workspace_bytes(dt, n, 0)
        ws = L.workspace(wsb, x.device)
        L.check(L.lib.tff_nblist_cell_list(dt, n, L.ptr(x), L.ptr(b), float(cutoff), L.ptr(rp), L.ptr(col),
                                           int(bool(include_self)), L.ptr(pairs), pairs.shape[0], L.ptr(npairs), 0,
                                           L.ptr(ws), ws.numel(), stream), "build_neighbor_list_cell_list")
    return npairs


def _capacity(n: int, max_npairs) -> int:
    m = int(max_npairs)
    return n * (n + 1) // 2 if m < 0 else m


def _nsq(coords, box, cutoff, max_npairs, rp, col, include_self):
    pairs = torch.empty((_capacity(coords.shape[0], max_npairs), 2), dtype=torch.int64, device=coords.device)
    return pairs, _nblist_out("nsquared", coords, box, cutoff, pairs, rp, col, include_self)


def _nsq_out(coords, box, cutoff, pairs, rp, col, include_self):
    return _nblist_out("nsquared", coords, box, cutoff, pairs, rp, col, include_self)


def _clist(coords, box, cutoff, max_npairs, rp, col, include_self):
    pairs = torch.empty((_capacity(coords.shape[0], max_npairs), 2), dtype=torch.int64, device=coords.device)
    return pairs, _nblist_out("cell_list", coords, box, cutoff, pairs, rp, col, include_self)


def _clist_out(coords, box, cutoff, pairs, rp, col, include_self):
    return pairs, _nblist_out("cell_list", coords, box, cutoff, pairs, rp, col, include_self)


_DEF.impl("build_neighbor_list_nsquared", _nsq, "CUDA")
_DEF.impl("build_neighbor_list_nsquared_out", _nsq_out, "CUDA")
_DEF.impl("build_neighbor_list_cell_list", _clist, "CUDA")
_DEF.impl("build_neighbor_list_cell_list_out", _clist_out, "CUDA")


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
# pair energy terms
# ---------------------------------------------------------------------------------------

def _pair_ws(x: torch.Tensor, ntypes: int = 0) -> torch.Tensor:
    return L.workspace(L.lib.tff_pairs_workspace_bytes(L.dtype_code(x.dtype), x.shape[0], ntypes), x.device)


def _empty_like_or_none(t, want):
    return torch.empty_like(t) if want else None


def nonbonded_forward(coords, pairs, box, sigma, epsilon, charges, coul_constant, cutoff, do_shift,
                      need=(False, False, False, False)):
    """Energy (1,) and optional dE/dx, dE/dsigma, dE/depsilon, dE/dq (``need`` in that order)."""
    L.require_cuda(coords, pairs, box, sigma, epsilon, charges)
    x = _c(coords.detach())
    dt = x.dtype
    p = _long(pairs.detach())
    b, s, e, q = (_c(t.detach(), dt) for t in (box, sigma, epsilon, charges))
    ene = torch.empty(1, dtype=dt, device=x.device)
    gx = _empty_like_or_none(x, need[0])
    gs = _empty_like_or_none(s, need[1])
    ge = _empty_like_or_none(e, need[2])
    gq = _empty_like_or_none(q, need[3])
    ws = _pair_ws(x)
    L.check(L.lib.tff_nonbonded_atom_pairs(L.dtype_code(dt), x.shape[0], L.ptr(x), p.shape[0], L.ptr(p), L.ptr(b),
                                           L.ptr(s), L.ptr(e), L.ptr(q), float(coul_constant), float(cutoff),
                                           int(bool(do_shift)), L.ptr(ene), L.ptr(gx), L.ptr(gs), L.ptr(ge), L.ptr(gq),
                                           L.ptr(ws), ws.numel(), L.stream_of(x)),
            "compute_nonbonded_energy_from_atom_pairs")
    return ene, gx, gs, ge, gq


class _NonbondedFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coords, pairs, box, sigma, epsilon, charges, coul_constant, cutoff, do_shift):
        ni = ctx.needs_input_grad
        ene, gx, gs, ge, gq = nonbonded_forward(coords, pairs, box, sigma, epsilon, charges, coul_constant, cutoff,
                                                do_shift, (ni[0], ni[3], ni[4], ni[5]))
        ctx.save_for_backward(gx, gs, ge, gq)
        return ene

    @staticmethod
    def backward(ctx, g):
        gx, gs, ge, gq = ctx.saved_tensors
        sc = lambda t: None if t is None else t * g
        return sc(gx), None, None, sc(gs), sc(ge), sc(gq), None, None, None


def _nonbonded_autograd(coords, pairs, box, sigma, epsilon, charges, coul_constant, cutoff, do_shift):
    return _NonbondedFn.apply(coords, pairs, box, sigma, epsilon, charges, coul_constant, cutoff, do_shift)


def _nonbonded_cuda(coords, pairs, box, sigma, epsilon, charges, coul_constant, cutoff, do_shift):
    return nonbonded_forward(coords, pairs, box, sigma, epsilon, charges, coul_constant, cutoff, do_shift)[0]


def _nonbonded_forces(coords, pairs, box, sigma, epsilon, charges, coul_constant, cutoff, forces):
    L.require_cuda(coords, pairs, box, sigma, epsilon, charges, forces)
    x = _c(coords.detach())
    dt = x.dtype
    if forces.dtype != dt or not forces.is_contiguous() or forces.shape != x.shape:
        raise RuntimeError("forces must be a contiguous tensor shaped and typed like coords")
    p = _long(pairs.detach())
    b, s, e, q = (_c(t.detach(), dt) for t in (box, sigma, epsilon, charges))
    ws = _pair_ws(x)
    L.check(L.lib.tff_nonbonded_forces_atom_pairs(L.dtype_code(dt), x.shape[0], L.ptr(x), p.shape[0], L.ptr(p),
                                                  L.ptr(b), L.ptr(s), L.ptr(e), L.ptr(q), float(coul_constant),
                                                  float(cutoff), L.ptr(forces), L.ptr(ws), ws.numel(),
                                                  L.stream_of(x)),
            "compute_nonbonded_forces_from_atom_pairs")


_DEF.impl("compute_nonbonded_energy_from_atom_pairs", _nonbonded_autograd, "AutogradCUDA")
_DEF.impl("compute_nonbonded_energy_from_atom_pairs", _nonbonded_cuda, "CUDA")
_DEF.impl("compute_nonbonded_forces_from_atom_pairs", _nonbonded_forces, "CUDA")


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


def coulomb_forward(coords, pairs, box, charges, coulomb_constant, cutoff, do_shift, need=(False, False)):
    L.require_cuda(coords, pairs, box, charges)
    x = _c(coords.detach())
    dt = x.dtype
    p = _long(pairs.detach())
    b, q = _c(box.detach(), dt), _c(charges.detach(), dt)
    ene = torch.empty(1, dtype=dt, device=x.device)
    gx = _empty_like_or_none(x, need[0])
    gq = _empty_like_or_none(q, need[1])
    ws = _pair_ws(x)
    L.check(L.lib.tff_coulomb_atom_pairs(L.dtype_code(dt), x.shape[0], L.ptr(x), p.shape[0], L.ptr(p), L.ptr(b),
                                         L.ptr(q), float(coulomb_constant), float(cutoff), int(bool(do_shift)),
                                         L.ptr(ene), L.ptr(gx), L.ptr(gq), L.ptr(ws), ws.numel(), L.stream_of(x)),
            "compute_coulomb_energy")
    return ene, gx, gq


class _CoulombFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coords, pairs, box, charges, coulomb_constant, cutoff, do_shift):
        ni = ctx.needs_input_grad
        ene, gx, gq = coulomb_forward(coords, pairs, box, charges, coulomb_constant, cutoff, do_shift, (ni[0], ni[3]))
        ctx.save_for_backward(gx, gq)
        return ene

    @staticmethod
    def backward(ctx, g):
        gx, gq = ctx.saved_tensors
        return (None if gx is None else gx * g), None, None, (None if gq is None else gq * g), None, None, None


_DEF.impl("compute_coulomb_energy", lambda *a: _CoulombFn.apply(*a), "AutogradCUDA")
_DEF.impl("compute_coulomb_energy", lambda *a: coulomb_forward(*a)[0], "CUDA")


def lj_forward(coords, pairs, box, sigma, epsilon, cutoff, atom_types, need=(False, False, False)):
    L.require_cuda(coords, pairs, box, sigma, epsilon, atom_types)
    x = _c(coords.detach())
    dt = x.dtype
    p = _long(pairs.detach())
    b, s, e = (_c(t.detach(), dt) for t in (box, sigma, epsilon))
    types = _long(atom_types)
    ntypes = 0
    if types is not None:
        if s.dim() != 2 or s.shape[0] != s.shape[1] or e.shape != s.shape:
            raise RuntimeError("with atom_types, sigma/epsilon must be (ntypes, ntypes) tables")
        ntypes = s.shape[0]
    elif s.shape[0] != p.shape[0] or e.shape[0] != p.shape[0]:
        raise RuntimeError("without atom_types, sigma/epsilon must be per pair, shape (P,)")
    ene = torch.empty((), dtype=dt, device=x.device)
    gx = _empty_like_or_none(x, need[0])
    gs = _empty_like_or_none(s, need[1])
    ge = _empty_like_or_none(e, need[2])
    ws = _pair_ws(x, ntypes)
    L.check(L.lib.tff_lennard_jones_atom_pairs(L.dtype_code(dt), x.shape[0], L.ptr(x), p.shape[0], L.ptr(p),
                                               L.ptr(b), L.ptr(s), L.ptr(e), float(cutoff), L.ptr(types), ntypes,
                                               L.ptr(ene), L.ptr(gx), L.ptr(gs), L.ptr(ge), L.ptr(ws), ws.numel(),
                                               L.stream_of(x)),
            "compute_lennard_jones_energy")
    return ene, gx, gs, ge


class _LJFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coords, pairs, box, sigma, epsilon, cutoff, atom_types):
        ni = ctx.needs_input_grad
        ene, gx, gs, ge = lj_forward(coords, pairs, box, sigma, epsilon, cutoff, atom_types, (ni[0], ni[3], ni[4]))
        ctx.save_for_backward(gx, gs, ge)
        return ene

    @staticmethod
    def backward(ctx, g):
        gx, gs, ge = ctx.saved_tensors
        sc = lambda t: None if t is None else t * g
        return sc(gx), None, None, sc(gs), sc(ge), None, None


def _vdw147(*args):
    raise NotImplementedError("the AMOEBA buffered 14-7 potential is outside the fixed-charge path")


_DEF.impl("compute_lennard_jones_energy", lambda *a: _LJFn.apply(*a), "AutogradCUDA")
_DEF.impl("compute_lennard_jones_energy", lambda *a: lj_forward(*a)[0], "CUDA")
_DEF.impl("compute_vdw_14_7_energy", _vdw147, "CUDA")
_DEF.impl("compute_vdw_14_7_energy", _vdw147, "AutogradCUDA")


def _rank0_only(p, t, what):
    if p is not None or t is not None:
        raise NotImplementedError(f"{what}: only rank 0 (point charges) is implemented")


def ewald_real_forward(coords, box, pairs, pairs_excl, q, cutoff, ewald_alpha, prefactor, need=(False, False)):
    L.require_cuda(coords, box, pairs, pairs_excl, q)
    x = _c(coords.detach())
    dt = x.dtype
    p = _long(pairs.detach())
    pe = _long(pairs_excl.detach()) if pairs_excl is not None else None
    b, qq = _c(box.detach(), dt), _c(q.detach(), dt)
    ene = torch.empty((), dtype=dt, device=x.device)
    gx = _empty_like_or_none(x, need[0])
    gq = _empty_like_or_none(qq, need[1])
    ws = _pair_ws(x)
    L.check(L.lib.tff_ewald_real_atom_pairs(L.dtype_code(dt), x.shape[0], L.ptr(x), L.ptr(b), p.shape[0], L.ptr(p),
                                            0 if pe is None else pe.shape[0], L.ptr(pe), L.ptr(qq), float(cutoff),
                                            float(ewald_alpha), float(prefactor), L.ptr(ene), L.ptr(gx), L.ptr(gq),
                                            L.ptr(ws), ws.numel(), L.stream_of(x)),
            "compute_multipolar_energy_from_atom_pairs")
    return ene, gx, gq


class _EwaldRealFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coords, box, pairs, pairs_excl, q, p, t, cutoff, ewald_alpha, prefactor):
        _rank0_only(p, t, "compute_multipolar_energy_from_atom_pairs")
        ni = ctx.needs_input_grad
        ene, gx, gq = ewald_real_forward(coords, box, pairs, pairs_excl, q, cutoff, ewald_alpha, prefactor,
                                         (ni[0], ni[4]))
        ctx.save_for_backward(gx, gq)
        return ene

    @staticmethod
    def backward(ctx, g):
        gx, gq = ctx.saved_tensors
        return (None if gx is None else gx * g), None, None, None, (None if gq is None else gq * g), \
            None, None, None, None, None


def _ewald_cuda(coords, box, pairs, pairs_excl, q, p, t, cutoff, ewald_alpha, prefactor):
    _rank0_only(p, t, "compute_multipolar_energy_from_atom_pairs")
    return ewald_real_forward(coords, box, pairs, pairs_excl, q, cutoff, ewald_alpha, prefactor)[0]


_DEF.impl("compute_multipolar_energy_from_atom_pairs", lambda *a: _EwaldRealFn.apply(*a), "AutogradCUDA")
_DEF.impl("compute_multipolar_energy_from_atom_pairs", _ewald_cuda, "CUDA")


# ---------------------------------------------------------------------------------------
# PME
# ---------------------------------------------------------------------------------------

class PmePlan:
    """Owns a libtffb200 PME plan (cuFFT R2C/C2R for one K and dtype on one device)."""

    def __init__(self, dtype: torch.dtype, K: int, device: torch.device):
        import ctypes

        self.K, self.dtype, self.device = int(K), dtype, device
        h = ctypes.c_void_p()
        with torch.cuda.device(device):
            L.check(L.lib.tff_pme_plan_create(L.dtype_code(dtype), self.K, ctypes.byref(h)), "tff_pme_plan_create")
        self.handle = h

    def workspace_bytes(self, natoms: int) -> int:
        return int(L.lib.tff_pme_workspace_bytes(self.handle, natoms))

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                L.lib.tff_pme_plan_destroy(h)
            except Exception:
                pass
            self.handle = None


_plans: dict = {}
_plans_lock = threading.Lock()


def get_pme_plan(dtype: torch.dtype, K: int, device: torch.device) -> PmePlan:
    key = (dtype, int(K), device.index if device.index is not None else torch.cuda.current_device())
    with _plans_lock:
        p = _plans.get(key)
        if p is None:
            p = PmePlan(dtype, K, torch.device("cuda", key[2]))
            _plans[key] = p
        return p


def pme_forward(coords, box, q, K, alpha, xmoduli, ymoduli, zmoduli, need=(False, False)):
    """Energy (0-d) and optional dE/dx, dE/dq = phi (self term included)."""
    L.require_cuda(coords, box, q, xmoduli, ymoduli, zmoduli)
    x = _c(coords.detach())
    dt = x.dtype
    b, qq = _c(box.detach(), dt), _c(q.detach(), dt)
    xm, ym, zm = (_c(m.detach(), dt) for m in (xmoduli, ymoduli, zmoduli))
    K = int(K)
    if xm.numel() != K or ym.numel() != K or zm.numel() != K // 2 + 1:
        raise RuntimeError("B-spline moduli must have K, K and K//2+1 entries")
    plan = get_pme_plan(dt, K, x.device)
    ene = torch.empty((), dtype=dt, device=x.device)
    gx = _empty_like_or_none(x, need[0])
    phi = _empty_like_or_none(qq, need[1])
    ws = L.workspace(plan.workspace_bytes(x.shape[0]), x.device)
    L.check(L.lib.tff_pme_long_range(plan.handle, x.shape[0], L.ptr(x), L.ptr(b), L.ptr(qq), float(alpha),
                                     L.ptr(xm), L.ptr(ym), L.ptr(zm), L.ptr(ene), L.ptr(phi), L.ptr(gx), L.ptr(ws),
                                     ws.numel(), L.stream_of(x)), "pme_long_range")
    return ene, gx, phi


class _PmeFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coords, box, q, p, t, K, alpha, xmoduli, ymoduli, zmoduli):
        _rank0_only(p, t, "pme_long_range")
        ni = ctx.needs_input_grad
        ene, gx, phi = pme_forward(coords, box, q, K, alpha, xmoduli, ymoduli, zmoduli, (ni[0], ni[2]))
        ctx.save_for_backward(gx, phi)
        return ene

    @staticmethod
    def backward(ctx, g):
        gx, phi = ctx.saved_tensors
        return (None if gx is None else gx * g), None, (None if phi is None else phi * g), \
            None, None, None, None, None, None, None


def _pme_cuda(coords, box, q, p, t, K, alpha, xmoduli, ymoduli, zmoduli):
    _rank0_only(p, t, "pme_long_range")
    return pme_forward(coords, box, q, K, alpha, xmoduli, ymoduli, zmoduli)[0]


_DEF.impl("pme_long_range", lambda *a: _PmeFn.apply(*a), "AutogradCUDA")
_DEF.impl("pme_long_range", _pme_cuda, "CUDA")


# ---------------------------------------------------------------------------------------
# bonded terms (AutogradCUDA + CUDA; forces variants CUDA)
# ---------------------------------------------------------------------------------------

def _bonded_ws(x: torch.Tensor, nterms: int) -> torch.Tensor:
    return L.workspace(L.lib.tff_bonded_workspace_bytes(L.dtype_code(x.dtype), x.shape[0], nterms), x.device)


def bonded_forward(angle: bool, coords, idx, p0, k, need=(False, False, False)):
    """Energy (0-d) of harmonic bonds (angle=False) or angles and the optional dE/dx,
    dE/dp0, dE/dk (``need`` in that order)."""
    L.require_cuda(coords, idx, p0, k)
    x = _c(coords.detach())
    dt = x.dtype
    ix = _long(idx.detach())
    if ix.dim() != 2 or ix.shape[1] != (3 if angle else 2):
        raise RuntimeError(f"{'angles' if angle else 'bonds'} must be an (M, {3 if angle else 2}) index tensor")
    a, kk = _c(p0.detach(), dt), _c(k.detach(), dt)
    ene = torch.empty((), dtype=dt, device=x.device)
    gx = _empty_like_or_none(x, need[0])
    gp = _empty_like_or_none(a, need[1])
    gk = _empty_like_or_none(kk, need[2])
    ws = _bonded_ws(x, ix.shape[0])
    fn = L.lib.tff_harmonic_angle if angle else L.lib.tff_harmonic_bond
    L.check(fn(L.dtype_code(dt), x.shape[0], L.ptr(x), ix.shape[0], L.ptr(ix), L.ptr(a), L.ptr(kk), L.ptr(ene),
               L.ptr(gx), L.ptr(gp), L.ptr(gk), L.ptr(ws), ws.numel(), L.stream_of(x)),
            "compute_harmonic_angle_energy" if angle else "compute_harmonic_bond_energy")
    return ene, gx, gp, gk


class _BondedFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, angle, coords, idx, p0, k):
        ni = ctx.needs_input_grad
        ene, gx, gp, gk = bonded_forward(angle, coords, idx, p0, k, (ni[1], ni[3], ni[4]))
        ctx.save_for_backward(gx, gp, gk)
        return ene

    @staticmethod
    def backward(ctx, g):
        gx, gp, gk = ctx.saved_tensors
        sc = lambda t: None if t is None else t * g
        return None, sc(gx), None, sc(gp), sc(gk)


def _bonded_forces(angle: bool, coords, idx, p0, k, forces):
    L.require_cuda(coords, idx, p0, k, forces)
    x = _c(coords.detach())
    dt = x.dtype
    if forces.dtype != dt or not forces.is_contiguous() or forces.shape != x.shape:
        raise RuntimeError("forces must be a contiguous tensor shaped and typed like coords")
    ix = _long(idx.detach())
    a, kk = _c(p0.detach(), dt), _c(k.detach(), dt)
    ws = _bonded_ws(x, ix.shape[0])
    fn = L.lib.tff_harmonic_angle_forces if angle else L.lib.tff_harmonic_bond_forces
    L.check(fn(L.dtype_code(dt), x.shape[0], L.ptr(x), ix.shape[0], L.ptr(ix), L.ptr(a), L.ptr(kk), L.ptr(forces),
               L.ptr(ws), ws.numel(), L.stream_of(x)),
            "compute_harmonic_angle_forces" if angle else "compute_harmonic_bond_forces")


def _angles_run(coords, angles, grad_theta=None):
    x = _c(coords.detach())
    ix = _long(angles.detach())
    if ix.dim() != 2 or ix.shape[1] != 3:
        raise RuntimeError("angles must be an (M, 3) index tensor")
    if grad_theta is None:
        theta = torch.empty(ix.shape[0], dtype=x.dtype, device=x.device)
        L.check(L.lib.tff_angles(L.dtype_code(x.dtype), x.shape[0], L.ptr(x), ix.shape[0], L.ptr(ix), L.ptr(theta),
                                 None, None, None, 0, L.stream_of(x)), "compute_angles")
        return theta
    gt = _c(grad_theta.detach(), x.dtype)
    gx = torch.empty_like(x)
    ws = _bonded_ws(x, ix.shape[0])
    L.check(L.lib.tff_angles(L.dtype_code(x.dtype), x.shape[0], L.ptr(x), ix.shape[0], L.ptr(ix), None, L.ptr(gt),
                             L.ptr(gx), L.ptr(ws), ws.numel(), L.stream_of(x)), "compute_angles backward")
    return gx


class _AnglesFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coords, angles):
        L.require_cuda(coords, angles)
        ctx.save_for_backward(coords, angles)
        return _angles_run(coords, angles)

    @staticmethod
    def backward(ctx, g):
        coords, angles = ctx.saved_tensors
        return _angles_run(coords, angles, g), None


_DEF.impl("compute_harmonic_bond_energy", lambda *a: _BondedFn.apply(False, *a), "AutogradCUDA")
_DEF.impl("compute_harmonic_bond_energy", lambda *a: bonded_forward(False, *a)[0], "CUDA")
_DEF.impl("compute_harmonic_bond_forces", lambda *a: _bonded_forces(False, *a), "CUDA")
_DEF.impl("compute_harmonic_angle_energy", lambda *a: _BondedFn.apply(True, *a), "AutogradCUDA")
_DEF.impl("compute_harmonic_angle_energy", lambda *a: bonded_forward(True, *a)[0], "CUDA")
_DEF.impl("compute_harmonic_angle_forces", lambda *a: _bonded_forces(True, *a), "CUDA")
_DEF.impl("compute_angles", lambda c, a: _AnglesFn.apply(c, a), "AutogradCUDA")
_DEF.impl("compute_angles", lambda c, a: (L.require_cuda(c, a), _angles_run(c, a))[1], "CUDA")
