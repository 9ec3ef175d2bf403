"""torchff_b200: sm_100a implementation of torchff's fixed-charge nonbonded energy/force path.

Importing the package loads libtffb200.so and registers the reference operator schemas
under ``torch.ops.torchff``. Module classes keep the reference names and signatures:
NeighborList, Nonbonded, Coulomb, Vdw, MultipolarInteraction (rank 0), PME (rank 0), PBC,
HarmonicBond, HarmonicAngle, Angles; FixedChargeSystem / FixedChargeNonbonded evaluate the
whole model (nonbonded, plus harmonic bonds and angles of flexible water) in one call;
TorchSimModel serves torch-sim states of one or many systems.
"""
from . import _lib  # noqa: F401  (fails loudly when the CUDA library is missing)
from . import ops  # noqa: F401
from .angle import Angles, HarmonicAngle, compute_angles, compute_harmonic_angle_energy
from .bond import HarmonicBond, compute_harmonic_bond_energy
from .coulomb import Coulomb, compute_coulomb_energy
from .multipoles import MultipolarInteraction, compute_multipolar_energy_from_atom_pairs
from .nblist import NeighborList, build_neighbor_list_cell_list, build_neighbor_list_nsquared
from .nblist import build_cluster_pairs, build_neighbor_list_cluster_pairs, decode_cluster_pairs
from .nonbonded import (Nonbonded, compute_nonbonded_energy_from_atom_pairs,
                        compute_nonbonded_energy_from_cluster_pairs, compute_nonbonded_forces_from_atom_pairs,
                        compute_nonbonded_forces_from_cluster_pairs)
from .pbc import PBC, applyPBC
from .pme import PME
from .serving import BatchEvaluator, Server, SystemSpec, autotune_atoms_per_cell
from .system import FixedChargeNonbonded, FixedChargeSystem
from .torchsim import Topology, TorchSimModel
from .vdw import Vdw, compute_lennard_jones_energy

__all__ = [
    "Coulomb", "compute_coulomb_energy", "MultipolarInteraction", "compute_multipolar_energy_from_atom_pairs",
    "NeighborList", "build_neighbor_list_cell_list", "build_neighbor_list_nsquared", "Nonbonded",
    "compute_nonbonded_energy_from_atom_pairs", "compute_nonbonded_forces_from_atom_pairs", "PBC", "applyPBC",
    "PME", "FixedChargeNonbonded", "FixedChargeSystem", "Vdw", "compute_lennard_jones_energy",
    "BatchEvaluator", "Server", "SystemSpec", "autotune_atoms_per_cell", "Angles", "HarmonicAngle",
    "compute_angles", "compute_harmonic_angle_energy", "HarmonicBond", "compute_harmonic_bond_energy",
    "build_cluster_pairs", "build_neighbor_list_cluster_pairs", "decode_cluster_pairs",
    "compute_nonbonded_energy_from_cluster_pairs", "compute_nonbonded_forces_from_cluster_pairs",
    "Topology", "TorchSimModel",
]
