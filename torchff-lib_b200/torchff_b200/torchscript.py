"""TorchScript route for C++ hosts (OpenMM-Torch ``TorchForce``, libtorch programs).

The reference reaches OpenMM by tracing ``Tip3pTorchFF`` built on its C++-registered ops
(``examples/tip3p/md.py:449-541``). Here the C++-registered piece is the TorchScript
custom class ``torch.classes.torchff_b200.System`` in ``libtffb200_torch.so``: a module
holding it can be scripted, saved with ``torch.jit.save`` and run by a process that only
loads that library (``torch.ops.load_library`` or, in C++, ``dlopen`` before
``torch::jit::load``). ``energy(coords, box)`` is differentiable in the coordinates, so
OpenMM-Torch gets forces from autograd; ``energy_forces`` returns them directly for
``setOutputsForces(True)``.
"""
from __future__ import annotations

import os

import torch
import torch.nn as nn

from ._build import torch_lib_path
from .system import COULOMB_PREFACTOR

_loaded = False


def library_path() -> str:
    """Path of libtffb200_torch.so (pass it to torch.ops.load_library in a C++ host's loader)."""
    return torch_lib_path()


def load_library() -> None:
    """Registers torch.classes.torchff_b200.System in this process (idempotent); raises if the
    library is not built."""
    global _loaded
    if _loaded:
        return
    p = torch_lib_path()
    if not os.path.exists(p):
        raise ImportError(f"{p} is not built; build it with `python torchff-lib_b200/torchff_b200/_build.py`")
    torch.ops.load_library(p)
    _loaded = True


def make_system(charges, sigma, epsilon, exclusions, cutoff: float, ewald_alpha: float, pme_grid: int,
                mixed: bool = True, coul_constant: float = COULOMB_PREFACTOR):
    """A torch.classes.torchff_b200.System (parameters as tensors or arrays)."""
    load_library()
    t = lambda a, dt: torch.as_tensor(a, dtype=dt).detach().cpu()
    return torch.classes.torchff_b200.System(
        t(charges, torch.float64), t(sigma, torch.float64), t(epsilon, torch.float64),
        t(exclusions if exclusions is not None else torch.zeros((0, 2)), torch.int64).reshape(-1, 2),
        float(cutoff), float(ewald_alpha), int(pme_grid), int(bool(mixed)), float(coul_constant))


class ScriptedTip3p(nn.Module):
    """Energy model forward(positions, box) -> 0-d energy, scriptable and savable: TIP3P
    nonbonded terms (+ the bonded terms of flexible water with ``flexible=True``)."""

    def __init__(self, wb, mixed: bool = True, flexible: bool = False):
        super().__init__()
        self.system = make_system(wb.charges, wb.sigma, wb.epsilon, wb.coulomb_exclusions, wb.cutoff, wb.alpha,
                                  wb.grid, mixed)
        if flexible:
            from .water import water_bonded_terms
            bt = water_bonded_terms(wb.n_waters)
            f64 = lambda a: torch.as_tensor(a, dtype=torch.float64)
            self.system.set_bonded(torch.as_tensor(bt.bonds), f64(bt.b0), f64(bt.kb), torch.as_tensor(bt.angles),
                                   f64(bt.th0), f64(bt.kth))

    def forward(self, positions: torch.Tensor, box: torch.Tensor) -> torch.Tensor:
        return self.system.energy(positions, box)
