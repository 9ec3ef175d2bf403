"""The oracle against the golden fixtures produced by the reference's own pure-torch code."""
import hashlib
import os

import numpy as np
import pytest

from conftest import GOLDEN, REPO
from oracle import oracle as O


def _rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_nblist_small_cases():
    g = np.load(os.path.join(GOLDEN, "nblist_small.npz"))
    for c in range(int(g["ncases"])):
        x = g[f"c{c}_coords"]
        n = x.shape[0]
        ex = g[f"c{c}_excl"]
        rp, col = O.exclusions_coo_to_csr(ex, n) if ex.shape[0] else (None, None)
        box = g[f"c{c}_box"] if bool(g[f"c{c}_periodic"]) else None
        p = O.nblist_pairs(x, box, float(g[f"c{c}_cutoff"]), rp, col, bool(g[f"c{c}_include_self"]))
        assert np.array_equal(O.canonical_pairs(p), g[f"c{c}_pairs"]), f"case {c}"


def test_water216_components():
    g = np.load(os.path.join(GOLDEN, "water216.npz"))
    n = g["coords"].shape[0]
    rp, col = O.exclusions_coo_to_csr(g["nblist_exclusions"], n)
    pairs = O.nblist_pairs(g["coords"], g["box"], float(g["cutoff"]), rp, col)
    assert pairs.shape[0] == int(g["npairs"])
    assert hashlib.sha256(pairs.tobytes()).hexdigest() == str(g["pairs_sha256"])
    e, gx, _, _ = O.lennard_jones(g["coords"], pairs, g["box"], g["sigma_table"], g["epsilon_table"],
                                  float(g["cutoff"]), g["atom_types"])
    assert abs(e - g["e_lj"]) <= 1e-12 * abs(g["e_lj"])
    assert _rel(gx, g["gx_lj"]) < 1e-12
    e, gx, gq = O.ewald_real(g["coords"], g["box"], pairs, g["charges"], float(g["cutoff"]), float(g["alpha"]),
                             138.935456, g["coulomb_exclusions"])
    assert abs(e - g["e_coul"]) <= 1e-12 * abs(g["e_coul"])
    assert _rel(gx, g["gx_coul"]) < 1e-12 and _rel(gq, g["gq_coul"]) < 1e-12
    e, gx, pot, _ = O.pme(g["coords"], g["box"], g["charges"], float(g["alpha"]), int(g["grid"]))
    assert abs(e - g["e_pme"]) <= 1e-12 * abs(g["e_pme"])
    assert _rel(gx, g["gx_pme"]) < 1e-11 and _rel(pot, g["gq_pme"]) < 1e-11


def test_pme_reference_input():
    g = np.load(os.path.join(GOLDEN, "pme_random300.npz"))
    e, gx, pot, _ = O.pme(g["coords"], g["box"], g["q"], float(g["alpha"]), int(g["K"]))
    assert abs(e - g["energy"]) <= 1e-12 * abs(g["energy"])
    assert _rel(gx, g["gx"]) < 1e-11 and _rel(pot, g["gq"]) < 1e-11


@pytest.mark.parametrize("tag,shift", [("shift", True), ("noshift", False)])
def test_nonbonded_lb(tag, shift):
    g = np.load(os.path.join(GOLDEN, "pairs_random.npz"))
    e, gx, gq, gs, ge = O.nonbonded(g["coords"], g["pairs"], g["box"], g["sigma"], g["epsilon"], g["q"],
                                    float(g["k"]), float(g["cutoff"]), shift)
    assert abs(e - g[f"{tag}_energy"]) <= 1e-12 * abs(g[f"{tag}_energy"])
    for a, b in ((gx, "gx"), (gq, "gq"), (gs, "gs"), (ge, "ge")):
        assert _rel(a, g[f"{tag}_{b}"]) < 1e-12


def test_lj_per_pair_and_types():
    g = np.load(os.path.join(GOLDEN, "pairs_random.npz"))
    e, gx, gs, ge = O.lennard_jones(g["coords"], g["pairs"], g["box"], g["lj_pair_sigma"], g["lj_pair_epsilon"],
                                    float(g["cutoff"]))
    assert abs(e - g["lj_pair_energy"]) <= 1e-12 * abs(g["lj_pair_energy"])
    assert _rel(gx, g["lj_pair_gx"]) < 1e-12 and _rel(gs, g["lj_pair_gs"]) < 1e-12
    assert _rel(ge, g["lj_pair_ge"]) < 1e-12
    e, gx, gs, ge = O.lennard_jones(g["coords"], g["pairs"], g["box"], g["lj_type_sigma"], g["lj_type_epsilon"],
                                    float(g["cutoff"]), g["lj_type_types"])
    assert abs(e - g["lj_type_energy"]) <= 1e-12 * abs(g["lj_type_energy"])
    assert _rel(gx, g["lj_type_gx"]) < 1e-12 and _rel(gs, g["lj_type_gs"]) < 1e-12
    assert _rel(ge, g["lj_type_ge"]) < 1e-12


def test_ewald_with_exclusions():
    g = np.load(os.path.join(GOLDEN, "pairs_random.npz"))
    e, gx, gq = O.ewald_real(g["coords"], g["box"], g["ewald_pairs"], g["q"], float(g["cutoff"]),
                             float(g["ewald_alpha"]), 138.935456, g["ewald_excl"])
    assert abs(e - g["ewald_energy"]) <= 1e-12 * abs(g["ewald_energy"])
    assert _rel(gx, g["ewald_gx"]) < 1e-12 and _rel(gq, g["ewald_gq"]) < 1e-12


def test_bspline_partition_of_unity():
    w = np.linspace(0, 1, 11, endpoint=False)
    vals = np.stack([O.bspline6(w + k)[0] for k in range(6)], 0)
    ders = np.stack([O.bspline6(w + k)[1] for k in range(6)], 0)
    assert np.allclose(vals.sum(0), 1.0, atol=1e-14)
    assert np.allclose(ders.sum(0), 0.0, atol=1e-13)


def test_bonded_water():
    """Harmonic bonds / angles and the angle values against the reference's pure-torch
    HarmonicBond, HarmonicAngle and compute_angles_ref (flexible 216-water box)."""
    g = np.load(os.path.join(GOLDEN, "bonded_water.npz"))
    e, gx, gb0, gk = O.harmonic_bond(g["coords"], g["bonds"], g["b0"], g["kb"])
    assert abs(e - float(g["bond_energy"])) <= 1e-13 * abs(float(g["bond_energy"]))
    assert _rel(gx, g["bond_gx"]) < 1e-12 and _rel(gb0, g["bond_gb0"]) < 1e-12 and _rel(gk, g["bond_gk"]) < 1e-12
    e, gx, gt, gk = O.harmonic_angle(g["coords"], g["angles"], g["th0"], g["kth"])
    assert abs(e - float(g["angle_energy"])) <= 1e-13 * abs(float(g["angle_energy"]))
    assert _rel(gx, g["angle_gx"]) < 1e-12 and _rel(gt, g["angle_gth0"]) < 1e-12 and _rel(gk, g["angle_gk"]) < 1e-12
    assert np.max(np.abs(O.angles(g["coords"], g["angles"]) - g["theta"])) < 1e-14


def test_large_box_oracle_matches_pair_list_oracle():
    """The cell-binned real-space energy, the sampled-atom real-space gradients and the
    sampled PME of the oracle (used for the 300,000-atom box) equal the pair-list oracle on
    the 3000-water box."""
    import sys

    sys.path.insert(0, os.path.join(REPO, "torchff-lib_b200"))
    from torchff_b200.water import water_box_3000

    wb = water_box_3000(0)
    ref = O.fixed_charge_energy(wb.coords, wb.box, wb.charges, wb.sigma_table, wb.epsilon_table, wb.atom_types,
                                wb.nblist_exclusions, wb.coulomb_exclusions, wb.cutoff, wb.alpha, wb.grid, 138.935456)
    e_real = O.real_space_cells(wb.coords, wb.box, wb.charges, wb.atom_types, wb.sigma_table, wb.epsilon_table,
                                wb.coulomb_exclusions, wb.cutoff, wb.alpha, 138.935456)
    assert abs(e_real - (ref["lj"] + ref["coul_real"])) < 1e-11 * (abs(ref["lj"]) + abs(ref["coul_real"]))
    subset = np.random.default_rng(5).choice(wb.natoms, 40, replace=False)
    e_pme, g_pme = O.pme_subset(wb.coords, wb.box, wb.charges, wb.alpha, wb.grid, subset)
    assert abs(e_pme - ref["pme_raw"]) < 1e-11 * abs(ref["pme_raw"])
    g_real = O.real_space_grad_subset(wb.coords, wb.box, wb.charges, wb.atom_types, wb.sigma_table,
                                      wb.epsilon_table, wb.coulomb_exclusions, wb.cutoff, wb.alpha, 138.935456, subset)
    g = g_real + 138.935456 * g_pme
    gref = ref["grad_coords"][subset]
    assert np.max(np.abs(g - gref)) < 1e-10 * np.max(np.abs(gref))
