"""torch-sim model interface over the fused evaluation.

The reference wraps its TIP3P model for torch-sim in ``Tip3pTorchSimModel``
(examples/tip3p/md_torchsim.py:98-140): positions and cell in Angstrom with the lattice
vectors as the cell's columns, energy in eV and forces in eV/Angstrom, while the force field
works in nm and kJ/mol. It evaluates exactly one periodic system and raises for
``state.n_systems != 1``. :class:`TorchSimModel` keeps that interface and those units and
evaluates a state of several systems (atoms ordered by system, as torch-sim lays them
out) in one batched launch per stage (:class:`~torchff_b200.serving.BatchEvaluator`),
with each system's own parameters, exclusions, PME grid and optional harmonic bonds and
angles (flexible water, examples/tip3p/model.py:105-106).

torch-sim itself is optional: when ``torch_sim`` is importable the class derives from its
``ModelInterface``; otherwise it is a ``torch.nn.Module`` with the same properties
(``device``, ``dtype``, ``compute_forces``, ``compute_stress``, ``memory_scales_with``).
Stress is not computed.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch
import torch.nn as nn

from .angle import compute_harmonic_angle_energy, compute_harmonic_angle_forces
from .bond import compute_harmonic_bond_energy, compute_harmonic_bond_forces
from .serving import MAX_ATOMS_PER_SYSTEM, BatchEvaluator, exclusion_table
from .system import COULOMB_PREFACTOR, FixedChargeSystem

KJMOL_PER_EV = 96.48533212331014  # kJ/mol per eV (examples/tip3p/md_torchsim.py:46)
NM_PER_ANGSTROM = 0.1

try:  # pragma: no cover - torch-sim is not part of this image
    from torch_sim.models.interface import ModelInterface as _Base
except ImportError:  # pragma: no cover
    _Base = nn.Module


@dataclass
class Topology:
    """Force-field parameters of one system (nm, kJ/mol, elementary charges)."""
    charges: np.ndarray          # (n,)
    sigma: np.ndarray            # (n,)
    epsilon: np.ndarray          # (n,)
    exclusions: np.ndarray       # (m, 2) int64, system-local atom indices
    pme_grid: int
    bonds: np.ndarray | None = None   # (nb, 2) int64, b0 (nb,), kb (nb,)
    b0: np.ndarray | None = None
    kb: np.ndarray | None = None
    angles: np.ndarray | None = None  # (na, 3) int64 (central atom in the middle), theta0, ktheta
    theta0: np.ndarray | None = None
    ktheta: np.ndarray | None = None

    @property
    def natoms(self) -> int:
        return int(np.asarray(self.charges).shape[0])

    @property
    def has_bonded(self) -> bool:
        return self.bonds is not None or self.angles is not None

    @classmethod
    def from_water_box(cls, wb, flexible: bool = False) -> "Topology":
        """TIP3P parameters of a ``torchff_b200.water.WaterBox``; ``flexible`` adds the O-H
        bonds and H-O-H angles of flexible TIP3P."""
        t = cls(np.asarray(wb.charges, np.float64), np.asarray(wb.sigma, np.float64),
                np.asarray(wb.epsilon, np.float64), np.asarray(wb.coulomb_exclusions, np.int64), int(wb.grid))
        if flexible:
            from .water import water_bonded_terms
            bt = water_bonded_terms(wb.n_waters)
            t.bonds, t.b0, t.kb, t.angles, t.theta0, t.ktheta = bt.bonds, bt.b0, bt.kb, bt.angles, bt.th0, bt.kth
        return t


def boxes_nm(cell: torch.Tensor) -> torch.Tensor:
    """(S, 3, 3) cells in Angstrom with lattice vectors as columns (ASE / torch-sim) ->
    (S, 3, 3) boxes in nm with lattice vectors as rows (torchff)."""
    return cell.transpose(-1, -2) * NM_PER_ANGSTROM


def system_offsets(system_idx: torch.Tensor | None, natoms: list[int]) -> np.ndarray:
    """Atom offsets of the systems, checking that ``system_idx`` lists every system's
    atoms contiguously and in order with the topology's atom counts."""
    off = np.concatenate([[0], np.cumsum(natoms)]).astype(np.int64)
    if system_idx is not None:
        idx = system_idx.detach().to("cpu", torch.int64).numpy()
        want = np.repeat(np.arange(len(natoms)), natoms)
        if idx.shape != want.shape or not np.array_equal(idx, want):
            raise ValueError("state atoms must be ordered by system with each system's topology atom count")
    return off


class TorchSimModel(_Base):
    """Energy and forces of a torch-sim ``SimState`` (one or several periodic systems).

    ``topologies``: one :class:`Topology` per system of the states this model will see
    (a single Topology serves single-system states). ``compute_dtype`` float32 selects
    mixed precision (FP32 arithmetic, fixed-point forces, FP64 energies), float64 full
    FP64; results come back in ``dtype`` (the state's dtype, float64 as in the reference).
    """

    def __init__(self, topologies: Topology | list[Topology], cutoff: float, ewald_alpha: float, *,
                 compute_dtype: torch.dtype = torch.float32, dtype: torch.dtype = torch.float64,
                 device: torch.device | str = "cuda", coul_constant: float = COULOMB_PREFACTOR,
                 compute_stress: bool = False):
        super().__init__()
        if compute_stress:
            raise NotImplementedError("stress is not computed")
        self.topologies = [topologies] if isinstance(topologies, Topology) else list(topologies)
        if not self.topologies:
            raise ValueError("at least one topology is needed")
        self.cutoff, self.ewald_alpha, self.coul_constant = float(cutoff), float(ewald_alpha), float(coul_constant)
        self.compute_dtype = compute_dtype
        self._device = torch.device(device)
        self._dtype = dtype
        self._compute_forces = True
        self._compute_stress = False
        self._memory_scales_with = "n_atoms"
        self._single: FixedChargeSystem | None = None
        self._batch: BatchEvaluator | None = None
        self._packed: dict | None = None
        self._bonded = None

    # ModelInterface properties
    @property
    def device(self) -> torch.device:
        return self._device

    @property
    def dtype(self) -> torch.dtype:
        return self._dtype

    @property
    def compute_forces(self) -> bool:
        return self._compute_forces

    @property
    def compute_stress(self) -> bool:
        return self._compute_stress

    @property
    def memory_scales_with(self) -> str:
        return self._memory_scales_with

    def _single_system(self) -> FixedChargeSystem:
        if self._single is None:
            t = self.topologies[0]
            s = FixedChargeSystem(t.charges, t.sigma, t.epsilon, t.exclusions, self.cutoff, self.ewald_alpha,
                                  t.pme_grid, self.coul_constant, dtype=self.compute_dtype, device=self._device)
            if t.has_bonded:
                s.set_bonded(t.bonds, t.b0, t.kb, t.angles, t.theta0, t.ktheta)
            self._single = s
        return self._single

    def _batch_setup(self) -> None:
        """The batched evaluator and the packed parameters of every system (built once)."""
        tops, dev, dt = self.topologies, self._device, self.compute_dtype
        if max(t.natoms for t in tops) > MAX_ATOMS_PER_SYSTEM:
            raise ValueError(f"batched systems are limited to {MAX_ATOMS_PER_SYSTEM} atoms each")
        natoms = np.array([t.natoms for t in tops], dtype=np.int64)
        grids = np.array([t.pme_grid for t in tops], dtype=np.int32)
        self._batch = BatchEvaluator(self.cutoff, self.ewald_alpha, dt, max_systems=len(tops),
                                     max_atoms=int(natoms.sum()), max_grid_points=int((grids.astype(np.int64) ** 3).sum()),
                                     coul_constant=self.coul_constant, device=dev)
        cat = lambda a: torch.from_numpy(np.concatenate(a).astype(np.float64)).to(dev, dt)  # noqa: E731
        self._packed = {
            "natoms": natoms, "pme_grid": grids,
            "charges": cat([t.charges for t in tops]), "sigma": cat([t.sigma for t in tops]),
            "epsilon": cat([t.epsilon for t in tops]),
            "excl": torch.from_numpy(np.concatenate([exclusion_table(t.natoms, t.exclusions) for t in tops])).to(dev),
            "energies": torch.empty(len(tops), dtype=torch.float64, device=dev),
            "forces": torch.empty((int(natoms.sum()), 3), dtype=dt, device=dev),
        }
        # bonded terms with batch-global atom indices, per system
        off = np.concatenate([[0], np.cumsum(natoms)])
        bonded = []
        for k, t in enumerate(tops):
            if not t.has_bonded:
                bonded.append(None)
                continue
            f = lambda a, d: None if a is None else torch.as_tensor(np.asarray(a), dtype=d, device=dev)  # noqa: E731
            bonded.append({
                "bonds": None if t.bonds is None else f(np.asarray(t.bonds, np.int64) + off[k], torch.int64),
                "b0": f(t.b0, dt), "kb": f(t.kb, dt),
                "angles": None if t.angles is None else f(np.asarray(t.angles, np.int64) + off[k], torch.int64),
                "theta0": f(t.theta0, dt), "ktheta": f(t.ktheta, dt)})
        self._bonded = bonded

    def forward(self, state, **kwargs) -> dict[str, torch.Tensor]:
        """``state``: positions (N, 3) Angstrom, cell (S, 3, 3) Angstrom (columns are lattice
        vectors), ``n_systems`` and ``system_idx`` (N,) as in torch-sim's ``SimState``.
        Returns energy (S,) in eV and forces (N, 3) in eV/Angstrom in the model dtype."""
        del kwargs
        nsys = int(getattr(state, "n_systems", state.cell.shape[0]))
        pos = state.positions
        cell = state.cell.reshape(-1, 3, 3)
        if nsys == 1 and len(self.topologies) == 1:
            return self._forward_single(pos, cell)
        if nsys != len(self.topologies):
            raise ValueError(f"state has {nsys} systems, the model {len(self.topologies)} topologies")
        return self._forward_batch(pos, cell, getattr(state, "system_idx", None))

    def _forward_single(self, pos: torch.Tensor, cell: torch.Tensor) -> dict[str, torch.Tensor]:
        s = self._single_system()
        out = s.evaluate(pos.detach() * NM_PER_ANGSTROM, boxes_nm(cell)[0])
        return {"energy": (out["energy"].to(torch.float64) / KJMOL_PER_EV).reshape(1).to(self._dtype),
                "forces": out["forces"].to(self._dtype) * (NM_PER_ANGSTROM / KJMOL_PER_EV)}

    def _forward_batch(self, pos: torch.Tensor, cell: torch.Tensor, system_idx) -> dict[str, torch.Tensor]:
        if self._batch is None:
            self._batch_setup()
        p = self._packed
        system_offsets(system_idx, [int(n) for n in p["natoms"]])
        dt = self.compute_dtype
        p["coords"] = (pos.detach().to(self._device) * NM_PER_ANGSTROM).to(dt).reshape(-1).contiguous()
        p["boxes"] = boxes_nm(cell.detach().to(self._device)).to(dt).reshape(-1).contiguous()
        self._batch.evaluate_packed(p)
        energy = p["energies"].clone()
        forces = p["forces"].clone()
        if any(b is not None for b in self._bonded):
            x = p["coords"].reshape(-1, 3)
            for k, b in enumerate(self._bonded):
                if b is None:
                    continue
                if b["bonds"] is not None:
                    energy[k] += compute_harmonic_bond_energy(x, b["bonds"], b["b0"], b["kb"]).to(torch.float64)
                    compute_harmonic_bond_forces(x, b["bonds"], b["b0"], b["kb"], forces)
                if b["angles"] is not None:
                    energy[k] += compute_harmonic_angle_energy(x, b["angles"], b["theta0"],
                                                               b["ktheta"]).to(torch.float64)
                    compute_harmonic_angle_forces(x, b["angles"], b["theta0"], b["ktheta"], forces)
        return {"energy": (energy / KJMOL_PER_EV).to(self._dtype),
                "forces": forces.to(self._dtype) * (NM_PER_ANGSTROM / KJMOL_PER_EV)}
