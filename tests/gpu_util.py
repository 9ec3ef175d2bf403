"""Shared helpers for the GPU parity tests."""
import numpy as np
import torch


def t(a, dtype=torch.float64, grad=False):
    x = torch.tensor(np.asarray(a), dtype=dtype, device="cuda")
    if grad:
        x.requires_grad_(True)
    return x


def rel_max(a, b):
    """max |a - b| / max |b| (a, b array-likes)."""
    a = a.detach().double().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a, float)
    b = b.detach().double().cpu().numpy() if isinstance(b, torch.Tensor) else np.asarray(b, float)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def rel_rms(a, b):
    a = a.detach().double().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a, float)
    b = b.detach().double().cpu().numpy() if isinstance(b, torch.Tensor) else np.asarray(b, float)
    return float(np.sqrt(np.mean((a - b) ** 2)) / np.sqrt(np.mean(b ** 2)))


def rel(a, b):
    return abs(float(a) - float(b)) / max(abs(float(b)), 1e-300)


def canon(pairs: torch.Tensor, npairs: torch.Tensor | None = None) -> np.ndarray:
    from oracle import oracle as O

    p = pairs.detach().cpu().numpy()
    if npairs is not None:
        p = p[: int(npairs.item())]
    return O.canonical_pairs(p)


def oracle_water(wb, coords=None, flexible: bool = False) -> dict:
    """The FP64 oracle of a water box's nonbonded model (LJ type tables + real-space Ewald with
    exclusion correction + 138.935456 x PME), plus the harmonic O-H bonds and H-O-H angles
    when ``flexible``: total energy, dE/dx, and the summed magnitudes of the terms (the scale
    of the mixed-precision energy tolerance)."""
    from oracle import oracle as O
    from torchff_b200.water import water_bonded_terms

    x = wb.coords if coords is None else coords
    ref = O.fixed_charge_energy(x, wb.box, wb.charges, wb.sigma_table, wb.epsilon_table, wb.atom_types,
                                wb.nblist_exclusions, wb.coulomb_exclusions, wb.cutoff, wb.alpha, wb.grid,
                                138.935456)
    e, g = ref["total"], ref["grad_coords"].copy()
    scale = abs(ref["lj"]) + abs(ref["coul_real"]) + abs(138.935456 * ref["pme_raw"])
    if flexible:
        bt = water_bonded_terms(wb.n_waters)
        eb, gb = O.harmonic_bond(x, bt.bonds, bt.b0, bt.kb)[:2]
        ea, ga = O.harmonic_angle(x, bt.angles, bt.th0, bt.kth)[:2]
        e, g, scale = e + eb + ea, g + gb + ga, scale + abs(eb) + abs(ea)
    return {"energy": e, "grad": g, "scale": scale}
