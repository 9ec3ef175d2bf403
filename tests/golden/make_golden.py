"""Generate the golden fixtures in this directory from the reference's own code.

Runs the reference's pure-torch path (THGLab/torchff-lib, ``torchff/*.py``) on CPU in
float64 with autograd and stores inputs and outputs as small ``.npz`` files:

* ``nblist_small.npz``   -- ``NeighborList(use_customized_ops=False)`` pair sets on seeded
                            random coordinates (periodic / open, with / without self pairs
                            and exclusions) (torchff/nblist.py:10-178);
* ``water216.npz``       -- the 216-water TIP3P box (648 atoms, L 1.8662 nm, rc 0.9,
                            K 20): neighbour-pair count and SHA-256 of the canonical pair
                            set, Lennard-Jones with type tables (torchff/vdw.py), rank-0
                            real-space Ewald with exclusion correction
                            (torchff/multipoles.py) and PME (torchff/pme.py,
                            torchff/pme_ref.py): energies and autograd gradients;
* ``pme_random300.npz``  -- rank-0 PME on the reference's own test input
                            ``tests/water/random_water_300.npz`` (alpha 0.26525, K 10);
* ``pairs_random.npz``   -- shifted Coulomb (torchff/coulomb.py:22-44) and LJ
                            (torchff/vdw.py:86-111) composed with Lorentz-Berthelot
                            combining, the fused term torchff/nonbonded.py:40-69 intends,
                            on seeded random atoms with per-atom parameters;
* ``bonded_water.npz``   -- harmonic bonds and angles (torchff/bond.py HarmonicBond,
                            torchff/angle.py HarmonicAngle and compute_angles_ref) of 216
                            flexible waters with distorted geometry and perturbed parameters:
                            energies, angles and autograd gradients.

The reference's compiled extension modules are replaced by empty stubs (the pure-torch
path never calls them). ``torchff/pme_ref.py`` switches the default device to CUDA at
import time, so the default device is reset to CPU afterwards.

Usage (needs a checkout of the reference; not run by the test-suite):
    python tests/golden/make_golden.py /path/to/torchff-lib [fixture names ...]
"""
from __future__ import annotations

import hashlib
import os
import sys
import types

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "torchff-lib_b200"))

from torchff_b200.water import water_bonded_terms, water_box_216, water_exclusions  # noqa: E402


def import_reference(ref_root: str):
    for name in ["torchff_bond", "torchff_angle", "torchff_nblist", "torchff_nb", "torchff_coulomb",
                 "torchff_vdw", "torchff_multipoles", "torchff_pme", "torchff_torsion",
                 "torchff_dispersion", "torchff_slater", "torchff_ewald"]:
        sys.modules[name] = types.ModuleType(name)
    sys.path.insert(0, ref_root)
    import torchff  # noqa: F401
    from torchff.multipoles import MultipolarInteraction
    from torchff.nblist import NeighborList
    from torchff.pme import PME
    from torchff.vdw import Vdw, compute_lennard_jones_energy_ref
    from torchff.coulomb import compute_coulomb_energy_ref
    from torchff.bond import HarmonicBond
    from torchff.angle import HarmonicAngle, compute_angles_ref
    torch.set_default_device("cpu")
    torch.set_default_dtype(torch.float64)
    return types.SimpleNamespace(
        NeighborList=NeighborList, MultipolarInteraction=MultipolarInteraction, PME=PME, Vdw=Vdw,
        lj_ref=compute_lennard_jones_energy_ref, coul_ref=compute_coulomb_energy_ref,
        HarmonicBond=HarmonicBond, HarmonicAngle=HarmonicAngle, angles_ref=compute_angles_ref,
    )


def canonical(pairs: np.ndarray) -> np.ndarray:
    hi = np.maximum(pairs[:, 0], pairs[:, 1])
    lo = np.minimum(pairs[:, 0], pairs[:, 1])
    q = np.stack([hi, lo], 1).astype(np.int64)
    return q[np.lexsort((q[:, 1], q[:, 0]))]


def sha(pairs: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(pairs, dtype=np.int64).tobytes()).hexdigest()


def gen_nblist_small(ref) -> dict:
    out = {}
    rng = np.random.default_rng(1234)
    cases = []
    for ci, (n, cutoff, periodic, include_self, with_excl) in enumerate([
        (50, 0.5, True, False, False),
        (100, 0.8, True, False, True),
        (100, 0.5, False, False, False),
        (80, 0.6, True, True, True),
        (64, 5.0, True, False, False),   # cutoff beyond the box: every pair
        (40, 0.0, True, False, False),   # zero cutoff: no pair
    ]):
        L = (n / 100.0) ** (1.0 / 3.0)
        coords = rng.random((n, 3)) * L
        box = np.eye(3) * L
        excl = None
        if with_excl:
            a = rng.integers(0, n, size=(n // 2,))
            b = rng.integers(0, n, size=(n // 2,))
            excl = np.stack([a, b], 1).astype(np.int64)
        nbl = ref.NeighborList(n, exclusions=None if excl is None else torch.tensor(excl),
                               include_self=include_self, use_customized_ops=False)
        pairs = nbl(torch.tensor(coords), torch.tensor(box) if periodic else None, cutoff).numpy()
        cases.append(ci)
        out[f"c{ci}_coords"] = coords
        out[f"c{ci}_box"] = box
        out[f"c{ci}_cutoff"] = np.float64(cutoff)
        out[f"c{ci}_periodic"] = np.bool_(periodic)
        out[f"c{ci}_include_self"] = np.bool_(include_self)
        out[f"c{ci}_excl"] = excl if excl is not None else np.zeros((0, 2), np.int64)
        out[f"c{ci}_pairs"] = canonical(pairs)
    out["ncases"] = np.int64(len(cases))
    return out


def gen_water216(ref) -> dict:
    wb = water_box_216(seed=0)
    n = wb.natoms
    coords = torch.tensor(wb.coords, requires_grad=True)
    box = torch.tensor(wb.box)
    q = torch.tensor(wb.charges, requires_grad=True)
    types_ = torch.tensor(wb.atom_types)
    nbl = ref.NeighborList(n, exclusions=torch.tensor(wb.nblist_exclusions), use_customized_ops=False)
    pairs = nbl(coords.detach(), box, wb.cutoff)
    pairs_np = canonical(pairs.numpy())
    lj = ref.Vdw("LennardJones", cutoff=wb.cutoff, use_customized_ops=False, use_type_pairs=True)
    sig_t = torch.tensor(wb.sigma_table)
    eps_t = torch.tensor(wb.epsilon_table)
    e_lj = lj(coords, pairs, box, sig_t, eps_t, wb.cutoff, atom_types=types_)
    g_lj = torch.autograd.grad(e_lj, coords)[0]
    coul = ref.MultipolarInteraction(rank=0, cutoff=wb.cutoff, ewald_alpha=wb.alpha,
                                     prefactor=138.935456, use_customized_ops=False)
    e_c = coul(coords, box, pairs, q, pairs_excl=torch.tensor(wb.coulomb_exclusions))
    gx_c, gq_c = torch.autograd.grad(e_c, (coords, q))
    pme = ref.PME(wb.alpha, wb.grid, 0, use_customized_ops=False)
    e_p = pme(coords, box, q)
    gx_p, gq_p = torch.autograd.grad(e_p, (coords, q))
    return {
        "coords": wb.coords, "box": wb.box, "charges": wb.charges, "atom_types": wb.atom_types,
        "sigma_table": wb.sigma_table, "epsilon_table": wb.epsilon_table,
        "nblist_exclusions": wb.nblist_exclusions, "coulomb_exclusions": wb.coulomb_exclusions,
        "cutoff": np.float64(wb.cutoff), "alpha": np.float64(wb.alpha), "grid": np.int64(wb.grid),
        "npairs": np.int64(pairs_np.shape[0]), "pairs_sha256": np.array(sha(pairs_np)),
        "e_lj": np.float64(e_lj.item()), "gx_lj": g_lj.numpy(),
        "e_coul": np.float64(e_c.item()), "gx_coul": gx_c.numpy(), "gq_coul": gq_c.numpy(),
        "e_pme": np.float64(e_p.item()), "gx_pme": gx_p.numpy(), "gq_pme": gq_p.numpy(),
    }


def gen_pme_random300(ref, ref_root: str) -> dict:
    d = np.load(os.path.join(ref_root, "tests", "water", "random_water_300.npz"))
    coords = torch.tensor(d["coords"], requires_grad=True)
    box = torch.tensor(d["box"])
    q = torch.tensor(d["q"], requires_grad=True)
    alpha = float(d["alpha"])
    K = int(d["max_hkl"])
    pme = ref.PME(alpha, K, 0, use_customized_ops=False)
    e = pme(coords, box, q)
    gx, gq = torch.autograd.grad(e, (coords, q))
    return {"coords": d["coords"], "box": d["box"], "q": d["q"], "alpha": np.float64(alpha),
            "K": np.int64(K), "energy": np.float64(e.item()), "gx": gx.numpy(), "gq": gq.numpy()}


def gen_pairs_random(ref) -> dict:
    rng = np.random.default_rng(99)
    n = 200
    # jittered 6x6x6 lattice, 200 of 216 sites: min separation ~0.14 nm keeps LJ finite
    L = 6 * 0.2
    s = np.arange(6)
    sx, sy, sz = np.meshgrid(s, s, s, indexing="ij")
    sites = (np.stack([sx.ravel(), sy.ravel(), sz.ravel()], 1) + 0.5) * 0.2
    coords_np = sites[rng.permutation(216)[:n]] + rng.uniform(-0.03, 0.03, (n, 3))
    box_np = np.eye(3) * L
    q_np = rng.standard_normal(n) * 0.5
    sig_np = rng.uniform(0.25, 0.35, n)
    eps_np = rng.uniform(0.1, 1.0, n)
    cutoff = 0.5
    nbl = ref.NeighborList(n, use_customized_ops=False)
    box = torch.tensor(box_np)
    pairs = nbl(torch.tensor(coords_np), box, 0.6)    # list longer than the cutoff on purpose
    coords = torch.tensor(coords_np, requires_grad=True)
    q = torch.tensor(q_np, requires_grad=True)
    sig = torch.tensor(sig_np, requires_grad=True)
    eps = torch.tensor(eps_np, requires_grad=True)
    out = {"coords": coords_np, "box": box_np, "q": q_np, "sigma": sig_np, "epsilon": eps_np,
           "cutoff": np.float64(cutoff), "pairs": pairs.numpy(), "k": np.float64(138.935456)}
    for shift in (True, False):
        e_c = ref.coul_ref(coords, pairs, box, q, 138.935456, cutoff, shift)
        from torchff.pbc import PBC
        dr = PBC()(coords[pairs[:, 0]] - coords[pairs[:, 1]], box)
        r = torch.norm(dr, dim=1)
        s_ij = 0.5 * (sig[pairs[:, 0]] + sig[pairs[:, 1]])
        e_ij = torch.sqrt(eps[pairs[:, 0]] * eps[pairs[:, 1]])
        e_lj = ref.lj_ref(r, s_ij, e_ij, sum=False)
        e_lj = torch.sum(torch.where(r <= cutoff, e_lj, 0.0))
        e = e_c + e_lj
        gx, gq, gs, ge = torch.autograd.grad(e, (coords, q, sig, eps))
        tag = "shift" if shift else "noshift"
        out[f"{tag}_energy"] = np.float64(e.item())
        out[f"{tag}_coul"] = np.float64(e_c.item())
        out[f"{tag}_gx"] = gx.numpy()
        out[f"{tag}_gq"] = gq.numpy()
        out[f"{tag}_gs"] = gs.numpy()
        out[f"{tag}_ge"] = ge.numpy()
    # per-pair LJ parameters and type tables (torchff/vdw.py:230-261)
    sig_p = rng.uniform(0.25, 0.35, pairs.shape[0])
    eps_p = rng.uniform(0.1, 1.0, pairs.shape[0])
    vdw = ref.Vdw("LennardJones", use_customized_ops=False)
    sp = torch.tensor(sig_p, requires_grad=True)
    ep = torch.tensor(eps_p, requires_grad=True)
    c2 = torch.tensor(coords_np, requires_grad=True)
    e = vdw(c2, pairs, box, sp, ep, cutoff)
    gx, gs, ge = torch.autograd.grad(e, (c2, sp, ep))
    out.update({"lj_pair_sigma": sig_p, "lj_pair_epsilon": eps_p, "lj_pair_energy": np.float64(e.item()),
                "lj_pair_gx": gx.numpy(), "lj_pair_gs": gs.numpy(), "lj_pair_ge": ge.numpy()})
    types_np = rng.integers(0, 3, n)
    st = rng.uniform(0.25, 0.35, (3, 3)); st = 0.5 * (st + st.T)
    et = rng.uniform(0.1, 1.0, (3, 3)); et = 0.5 * (et + et.T)
    vdw_t = ref.Vdw("LennardJones", use_customized_ops=False, use_type_pairs=True)
    stt = torch.tensor(st, requires_grad=True)
    ett = torch.tensor(et, requires_grad=True)
    c3 = torch.tensor(coords_np, requires_grad=True)
    e = vdw_t(c3, pairs, box, stt, ett, cutoff, atom_types=torch.tensor(types_np))
    gx, gs, ge = torch.autograd.grad(e, (c3, stt, ett))
    out.update({"lj_type_types": types_np, "lj_type_sigma": st, "lj_type_epsilon": et,
                "lj_type_energy": np.float64(e.item()), "lj_type_gx": gx.numpy(),
                "lj_type_gs": gs.numpy(), "lj_type_ge": ge.numpy()})
    # rank-0 Ewald real space with an exclusion list (torchff/multipoles.py:244-341)
    excl = pairs[:: 7].clone()
    keep = torch.ones(pairs.shape[0], dtype=torch.bool)
    keep[:: 7] = False
    pl = pairs[keep]
    mi = ref.MultipolarInteraction(rank=0, cutoff=cutoff, ewald_alpha=3.0, prefactor=138.935456,
                                   use_customized_ops=False)
    c4 = torch.tensor(coords_np, requires_grad=True)
    q4 = torch.tensor(q_np, requires_grad=True)
    e = mi(c4, box, pl, q4, pairs_excl=excl)
    gx, gq = torch.autograd.grad(e, (c4, q4))
    out.update({"ewald_pairs": pl.numpy(), "ewald_excl": excl.numpy(), "ewald_alpha": np.float64(3.0),
                "ewald_energy": np.float64(e.item()), "ewald_gx": gx.numpy(), "ewald_gq": gq.numpy()})
    return out


def gen_bonded_water(ref) -> dict:
    wb = water_box_216(seed=3)
    bt = water_bonded_terms(wb.n_waters)
    rng = np.random.default_rng(7)
    coords_np = wb.coords + rng.normal(0.0, 0.006, wb.coords.shape)
    b0_np = bt.b0 * (1.0 + rng.uniform(-0.03, 0.03, bt.b0.shape))
    kb_np = bt.kb * (1.0 + rng.uniform(-0.1, 0.1, bt.kb.shape))
    th0_np = bt.th0 + rng.uniform(-0.05, 0.05, bt.th0.shape)
    kth_np = bt.kth * (1.0 + rng.uniform(-0.1, 0.1, bt.kth.shape))
    x = torch.tensor(coords_np, requires_grad=True)
    b0 = torch.tensor(b0_np, requires_grad=True)
    kb = torch.tensor(kb_np, requires_grad=True)
    e_b = ref.HarmonicBond(use_customized_ops=False)(x, torch.tensor(bt.bonds), b0, kb)
    gx_b, gb0, gkb = torch.autograd.grad(e_b, (x, b0, kb))
    th0 = torch.tensor(th0_np, requires_grad=True)
    kth = torch.tensor(kth_np, requires_grad=True)
    x2 = torch.tensor(coords_np, requires_grad=True)
    e_a = ref.HarmonicAngle(use_customized_ops=False)(x2, torch.tensor(bt.angles), th0, kth)
    gx_a, gth0, gkth = torch.autograd.grad(e_a, (x2, th0, kth))
    theta = ref.angles_ref(torch.tensor(coords_np), torch.tensor(bt.angles))
    return {"coords": coords_np, "bonds": bt.bonds, "b0": b0_np, "kb": kb_np, "angles": bt.angles,
            "th0": th0_np, "kth": kth_np, "bond_energy": np.float64(e_b.item()), "bond_gx": gx_b.numpy(),
            "bond_gb0": gb0.numpy(), "bond_gk": gkb.numpy(), "angle_energy": np.float64(e_a.item()),
            "angle_gx": gx_a.numpy(), "angle_gth0": gth0.numpy(), "angle_gk": gkth.numpy(),
            "theta": theta.numpy()}


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TORCHFF_REFERENCE", "")
    if not ref_root or not os.path.isdir(ref_root):
        raise SystemExit("usage: make_golden.py /path/to/torchff-lib")
    ref = import_reference(ref_root)
    gens = {"nblist_small": lambda: gen_nblist_small(ref), "water216": lambda: gen_water216(ref),
            "pme_random300": lambda: gen_pme_random300(ref, ref_root), "pairs_random": lambda: gen_pairs_random(ref),
            "bonded_water": lambda: gen_bonded_water(ref)}
    names = sys.argv[2:] or list(gens)
    for name in names:
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **gens[name]())
    print("golden fixtures written to", HERE, names)


if __name__ == "__main__":
    main()
