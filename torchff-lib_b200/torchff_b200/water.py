"""Seeded synthetic rigid TIP3P water boxes.

The reference builds its TIP3P systems from OpenMM-minimised PDB files
(``examples/tip3p/md.py:243-330``); OpenMM is not available here, so boxes are
generated synthetically with the same force-field parameters:

* rigid water, O-H 0.09572 nm, H-O-H 104.52 degrees;
* charges O -0.834 e, H +0.417 e;
* Lennard-Jones on O only (sigma 0.315061 nm, epsilon 0.636386 kJ/mol); H has
  epsilon 0 (sigma 1.0 nm, the value of OpenMM's tip3p.xml, which never enters an
  energy because epsilon_ij = 0 for every pair involving H);
* intramolecular pairs excluded: the neighbour list excludes all 9 ordered pairs of
  each water including self (``examples/tip3p/md.py:141-149``) and the real-space
  Ewald exclusion correction runs over the 3 unique intramolecular pairs
  (``examples/tip3p/md.py:152-158``).

Waters sit on a cubic lattice (``sites_per_dim`` sites per edge, spacing L/n), the
first ``n_waters`` sites of a seeded permutation are occupied, the oxygen is jittered
by U(-jitter, jitter) per coordinate and the molecule gets a uniformly random
orientation. Everything is numpy so the oracle, the tests and the benchmark share one
construction.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

COULOMB_PREFACTOR = 138.935456  # kJ mol^-1 nm e^-2, examples/tip3p/model.py:22
OH_BOND = 0.09572
HOH_ANGLE_DEG = 104.52
Q_O, Q_H = -0.834, 0.417
SIGMA_O, EPS_O = 0.315061, 0.636386
SIGMA_H, EPS_H = 1.0, 0.0


def ewald_alpha_from_tolerance(cutoff: float, tol: float = 5e-4) -> float:
    """alpha = sqrt(-ln(2 tol)) / rc, the OpenMM/torchff rule for the real-space tail."""
    return math.sqrt(-math.log(2.0 * tol)) / cutoff


@dataclass
class WaterBox:
    coords: np.ndarray          # (N, 3) float64, nm
    box: np.ndarray             # (3, 3) float64, rows are box vectors
    charges: np.ndarray         # (N,)
    sigma: np.ndarray           # (N,) per-atom sigma
    epsilon: np.ndarray         # (N,) per-atom epsilon
    atom_types: np.ndarray      # (N,) int64, 0 = O, 1 = H
    sigma_table: np.ndarray     # (2, 2) Lorentz-Berthelot type table
    epsilon_table: np.ndarray   # (2, 2)
    nblist_exclusions: np.ndarray  # (9 n, 2) int64, all intra-water ordered pairs incl. self
    coulomb_exclusions: np.ndarray  # (3 n, 2) int64, O-H1, O-H2, H1-H2
    cutoff: float
    alpha: float
    grid: int
    n_waters: int
    meta: dict = field(default_factory=dict)

    @property
    def natoms(self) -> int:
        return self.coords.shape[0]


def _random_rotations(rng: np.random.Generator, n: int) -> np.ndarray:
    """Uniform random rotation matrices from normalised Gaussian quaternions."""
    q = rng.standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    r = np.empty((n, 3, 3))
    r[:, 0, 0] = 1 - 2 * (y * y + z * z)
    r[:, 0, 1] = 2 * (x * y - z * w)
    r[:, 0, 2] = 2 * (x * z + y * w)
    r[:, 1, 0] = 2 * (x * y + z * w)
    r[:, 1, 1] = 1 - 2 * (x * x + z * z)
    r[:, 1, 2] = 2 * (y * z - x * w)
    r[:, 2, 0] = 2 * (x * z - y * w)
    r[:, 2, 1] = 2 * (y * z + x * w)
    r[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return r


def water_exclusions(n_waters: int) -> tuple[np.ndarray, np.ndarray]:
    """(nblist exclusions incl. self, Ewald-correction pairs) for n rigid waters."""
    base = 3 * np.arange(n_waters, dtype=np.int64)
    a = np.arange(3)
    ii, jj = np.meshgrid(a, a, indexing="ij")
    nb = (base[:, None, None] + np.stack([ii.ravel(), jj.ravel()], 1)[None]).reshape(-1, 2)
    tri = np.array([[0, 1], [0, 2], [1, 2]], dtype=np.int64)
    coul = (base[:, None, None] + tri[None]).reshape(-1, 2)
    return nb.astype(np.int64), coul.astype(np.int64)


# Flexible TIP3P bonded parameters (the harmonic terms of OpenMM's tip3p-flexible force field):
# E_bond = 1/2 K_BOND (r - OH_BOND)^2, E_angle = 1/2 K_ANGLE (theta - HOH_ANGLE)^2.
K_BOND = 462750.4        # kJ mol^-1 nm^-2
K_ANGLE = 836.8          # kJ mol^-1 rad^-2


@dataclass
class WaterBonded:
    bonds: np.ndarray    # (2 n, 2) int64: O-H1, O-H2 per water
    b0: np.ndarray       # (2 n,) nm
    kb: np.ndarray       # (2 n,) kJ/mol/nm^2
    angles: np.ndarray   # (n, 3) int64: H1-O-H2 (O central)
    th0: np.ndarray      # (n,) rad
    kth: np.ndarray      # (n,) kJ/mol/rad^2


def water_bonded_terms(n_waters: int) -> WaterBonded:
    """Harmonic O-H bonds and H-O-H angles of n flexible TIP3P waters (atoms O, H1, H2)."""
    base = 3 * np.arange(n_waters, dtype=np.int64)
    bonds = np.stack([np.stack([base, base + 1], 1), np.stack([base, base + 2], 1)], 1).reshape(-1, 2)
    angles = np.stack([base + 1, base, base + 2], 1)
    return WaterBonded(bonds=bonds, b0=np.full(2 * n_waters, OH_BOND), kb=np.full(2 * n_waters, K_BOND),
                       angles=angles, th0=np.full(n_waters, math.radians(HOH_ANGLE_DEG)),
                       kth=np.full(n_waters, K_ANGLE))


def make_water_box(
    n_waters: int,
    box_len: float,
    sites_per_dim: int,
    cutoff: float,
    grid: int,
    seed: int = 0,
    jitter: float = 0.02,
    ewald_tol: float = 5e-4,
) -> WaterBox:
    if n_waters > sites_per_dim ** 3:
        raise ValueError("more waters than lattice sites")
    rng = np.random.default_rng(seed)
    spacing = box_len / sites_per_dim
    s = np.arange(sites_per_dim)
    sx, sy, sz = np.meshgrid(s, s, s, indexing="ij")
    sites = (np.stack([sx.ravel(), sy.ravel(), sz.ravel()], 1) + 0.5) * spacing
    order = rng.permutation(sites.shape[0])[:n_waters]
    oxy = sites[order] + rng.uniform(-jitter, jitter, size=(n_waters, 3))
    half = math.radians(HOH_ANGLE_DEG) / 2.0
    local = np.array(
        [
            [0.0, 0.0, 0.0],
            [OH_BOND * math.sin(half), OH_BOND * math.cos(half), 0.0],
            [-OH_BOND * math.sin(half), OH_BOND * math.cos(half), 0.0],
        ]
    )
    rot = _random_rotations(rng, n_waters)
    mol = np.einsum("nij,aj->nai", rot, local) + oxy[:, None, :]
    coords = mol.reshape(-1, 3)
    natoms = coords.shape[0]
    types = np.tile(np.array([0, 1, 1], dtype=np.int64), n_waters)
    charges = np.where(types == 0, Q_O, Q_H).astype(np.float64)
    sigma = np.where(types == 0, SIGMA_O, SIGMA_H).astype(np.float64)
    eps = np.where(types == 0, EPS_O, EPS_H).astype(np.float64)
    sig_t = np.array([SIGMA_O, SIGMA_H])
    eps_t = np.array([EPS_O, EPS_H])
    sigma_table = 0.5 * (sig_t[:, None] + sig_t[None, :])
    epsilon_table = np.sqrt(eps_t[:, None] * eps_t[None, :])
    nb_excl, coul_excl = water_exclusions(n_waters)
    box = np.eye(3) * box_len
    assert natoms == 3 * n_waters
    return WaterBox(
        coords=coords,
        box=box,
        charges=charges,
        sigma=sigma,
        epsilon=eps,
        atom_types=types,
        sigma_table=sigma_table,
        epsilon_table=epsilon_table,
        nblist_exclusions=nb_excl,
        coulomb_exclusions=coul_excl,
        cutoff=float(cutoff),
        alpha=ewald_alpha_from_tolerance(cutoff, ewald_tol),
        grid=int(grid),
        n_waters=n_waters,
        meta={"seed": seed, "sites_per_dim": sites_per_dim, "jitter": jitter},
    )


# The workloads: 216 waters (648 atoms), 3000 waters (9000 atoms) and 100,000 waters
# (300,000 atoms) with the cutoffs and PME grids used throughout the tests and bench.
def water_box_216(seed: int = 0) -> WaterBox:
    return make_water_box(216, 1.8662, 6, cutoff=0.9, grid=20, seed=seed)


def water_box_3000(seed: int = 0) -> WaterBox:
    return make_water_box(3000, 4.482, 15, cutoff=1.0, grid=48, seed=seed)


def water_box_100k(seed: int = 0) -> WaterBox:
    return make_water_box(100_000, 14.42, 47, cutoff=1.0, grid=144, seed=seed)


def serving_water_box(n_waters: int, seed: int, density: float = 33.4,
                      cutoff: float = 0.9, spacing: float = 0.1) -> WaterBox:
    """Serving request box: L = (n / density)^(1/3), grid K = ceil(L / spacing)."""
    box_len = (n_waters / density) ** (1.0 / 3.0)
    sites = int(math.ceil(n_waters ** (1.0 / 3.0) - 1e-9))
    grid = int(math.ceil(box_len / spacing))
    return make_water_box(n_waters, box_len, sites, cutoff=cutoff, grid=grid, seed=seed)


def perturbed_frames(wb: WaterBox, n_frames: int, sigma: float, seed: int) -> np.ndarray:
    """(n_frames, N, 3): frame 0 is the base box, the rest add seeded N(0, sigma) noise."""
    rng = np.random.default_rng(seed)
    frames = np.repeat(wb.coords[None], n_frames, axis=0).copy()
    if n_frames > 1:
        frames[1:] += rng.normal(0.0, sigma, size=frames[1:].shape)
    return frames


def force_matching_parameters(wb: WaterBox, seed: int, noise: float = 0.05) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Per-atom (charges, sigma, epsilon) for force matching: TIP3P charges with seeded
    uniform +-`noise` relative noise, shifted back to a neutral total; sigma and epsilon
    are the TIP3P per-atom values."""
    rng = np.random.default_rng(seed)
    q = wb.charges * (1.0 + rng.uniform(-noise, noise, wb.natoms))
    q -= q.mean()
    return q, wb.sigma.copy(), wb.epsilon.copy()
