"""The drop-in operators for C++ hosts. libtffb200_torch.so registers the reference's
operator schemas (torch.ops.torchff.*) in C++, so they exist in a process that never imports
torchff_b200. A model in the shape of the reference's Tip3pTorchFF (examples/tip3p/model.py:
28-133: NeighborList + HarmonicBond + HarmonicAngle + Vdw type tables + rank-0
MultipolarInteraction with pairs_excl + 138.935456 x PME), built from this package's drop-in
modules and traced the way examples/tip3p/md.py:449-471 traces it for OpenMM-Torch's
TorchForce, runs in such a process with the energy and forces of the in-process trace and of
the FP64 oracle."""
import subprocess
import sys
import textwrap

import numpy as np
import pytest
import torch

from gpu_util import oracle_water, rel_rms

# The reference's registered schemas (csrc/*/*_interface.cpp), as torch prints them.
REFERENCE_SCHEMAS = {
    "build_neighbor_list_nsquared": "(Tensor coords, Tensor? box, Scalar cutoff, Scalar max_npairs, Tensor? excl_row_ptr, Tensor? excl_col_indices, bool include_self) -> (Tensor, Tensor)",
    "build_neighbor_list_nsquared_out": "(Tensor coords, Tensor? box, Scalar cutoff, Tensor(a!) pairs, Tensor? excl_row_ptr, Tensor? excl_col_indices, bool include_self) -> Tensor",
    "build_neighbor_list_cell_list": "(Tensor coords, Tensor? box, Scalar cutoff, Scalar max_npairs, Tensor? excl_row_ptr, Tensor? excl_col_indices, bool include_self) -> (Tensor, Tensor)",
    "build_neighbor_list_cell_list_out": "(Tensor coords, Tensor? box, Scalar cutoff, Tensor(a!) pairs, Tensor? excl_row_ptr, Tensor? excl_col_indices, bool include_self) -> (Tensor, Tensor)",
    "compute_nonbonded_energy_from_atom_pairs": "(Tensor coords, Tensor pairs, Tensor box, Tensor sigma, Tensor epsilon, Tensor charges, Scalar coul_constant, Scalar cutoff, bool do_shift) -> Tensor",
    "compute_nonbonded_forces_from_atom_pairs": "(Tensor coords, Tensor pairs, Tensor box, Tensor sigma, Tensor epsilon, Tensor charges, Scalar coul_constant, Scalar cutoff, Tensor forces) -> ()",
    "compute_coulomb_energy": "(Tensor coords, Tensor pairs, Tensor box, Tensor charges, Scalar coulomb_constant, Scalar cutoff, bool do_shift) -> Tensor",
    "compute_lennard_jones_energy": "(Tensor coords, Tensor pairs, Tensor box, Tensor sigma, Tensor epsilon, Scalar cutoff, Tensor? atom_types) -> Tensor",
    "compute_vdw_14_7_energy": "(Tensor coords, Tensor pairs, Tensor box, Tensor radius, Tensor epsilon, Scalar cutoff, Tensor? atom_types) -> Tensor",
    "compute_multipolar_energy_from_atom_pairs": "(Tensor coords, Tensor box, Tensor pairs, Tensor? pairs_excl, Tensor q, Tensor? p, Tensor? t, Scalar cutoff, Scalar ewald_alpha, Scalar prefactor) -> Tensor",
    "compute_harmonic_bond_energy": "(Tensor coords, Tensor pairs, Tensor b0, Tensor k) -> Tensor",
    "compute_harmonic_bond_forces": "(Tensor coords, Tensor pairs, Tensor b0, Tensor k, Tensor(a!) forces) -> ()",
    "compute_harmonic_angle_energy": "(Tensor coords, Tensor angles, Tensor theta0, Tensor k) -> Tensor",
    "compute_harmonic_angle_forces": "(Tensor coords, Tensor angles, Tensor theta0, Tensor k, Tensor(a!) forces) -> ()",
    "compute_angles": "(Tensor coords, Tensor angles) -> Tensor",
    "pme_long_range": "(Tensor coords, Tensor box, Tensor q, Tensor? p, Tensor? t, Scalar K, Scalar alpha, Tensor xmoduli, Tensor ymoduli, Tensor zmoduli) -> Tensor",
}


def _library_path() -> str:
    from torchff_b200._build import torch_lib_path

    return torch_lib_path()


def test_schemas_register_in_a_process_without_the_package():
    code = textwrap.dedent(f"""
        import json, sys, torch
        torch.ops.load_library({_library_path()!r})
        out = {{n: str(getattr(torch.ops.torchff, n).default._schema) for n in {sorted(REFERENCE_SCHEMAS)!r}}}
        out["_package_imported"] = any(m.startswith("torchff_b200") for m in sys.modules)
        print(json.dumps(out))
    """)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd="/")
    assert r.returncode == 0, r.stderr[-2000:]
    import json

    got = json.loads(r.stdout.strip().splitlines()[-1])
    assert got.pop("_package_imported") is False
    for name, sig in REFERENCE_SCHEMAS.items():
        assert got[name] == f"torchff::{name}{sig}", name


class Tip3pModel(torch.nn.Module):
    """The composition of the reference's Tip3pTorchFF.energy_components on this package's
    drop-in modules (nsquared neighbour list with the intramolecular exclusions, padded
    pairs), in FP32 as the reference traces it for OpenMM."""

    def __init__(self, wb, flexible: bool):
        from torchff_b200 import PME, MultipolarInteraction, NeighborList, Vdw
        from torchff_b200.angle import HarmonicAngle
        from torchff_b200.bond import HarmonicBond
        from torchff_b200.water import water_bonded_terms

        super().__init__()
        f32 = torch.float32
        self.flexible = flexible
        self.cutoff = float(wb.cutoff)
        self.register_buffer("charges", torch.tensor(wb.charges, dtype=f32))
        self.register_buffer("sigma", torch.tensor(wb.sigma_table, dtype=f32))
        self.register_buffer("epsilon", torch.tensor(wb.epsilon_table, dtype=f32))
        self.register_buffer("atom_types", torch.tensor(wb.atom_types, dtype=torch.int64))
        self.register_buffer("coulomb_excl_pairs", torch.tensor(wb.coulomb_exclusions, dtype=torch.int64))
        bt = water_bonded_terms(wb.n_waters)
        self.register_buffer("bonds", torch.tensor(bt.bonds))
        self.register_buffer("b0", torch.tensor(bt.b0, dtype=f32))
        self.register_buffer("kb", torch.tensor(bt.kb, dtype=f32))
        self.register_buffer("angles", torch.tensor(bt.angles))
        self.register_buffer("th0", torch.tensor(bt.th0, dtype=f32))
        self.register_buffer("kth", torch.tensor(bt.kth, dtype=f32))
        self.bond = HarmonicBond(use_customized_ops=True)
        self.angle = HarmonicAngle(use_customized_ops=True)
        self.lj = Vdw("LennardJones", cutoff=wb.cutoff, use_customized_ops=True, use_type_pairs=True)
        self.coul = MultipolarInteraction(0, wb.cutoff, ewald_alpha=wb.alpha, prefactor=138.935456,
                                          use_customized_ops=True)
        self.pme = PME(alpha=wb.alpha, max_hkl=wb.grid, rank=0, use_customized_ops=True)
        self.nblist = NeighborList(wb.natoms, exclusions=torch.tensor(wb.nblist_exclusions),
                                   use_customized_ops=True, algorithm="nsquared")
        self.max_npairs = int(wb.natoms * 4 / 3 * 3.1416 * wb.cutoff ** 3 * 100 / 2 * 1.2)

    def forward(self, coords, box):
        pairs = self.nblist(coords, box, self.cutoff, self.max_npairs, padding=True)[0]
        e = (self.lj(coords, pairs, box, self.sigma, self.epsilon, self.cutoff, atom_types=self.atom_types)
             + self.coul(coords, box, pairs, self.charges, pairs_excl=self.coulomb_excl_pairs)
             + self.pme(coords, box, self.charges) * 138.935456)
        if self.flexible:
            e = e + self.bond(coords, self.bonds, self.b0, self.kb) + self.angle(coords, self.angles, self.th0,
                                                                                self.kth)
        return e


@pytest.mark.gpu
@pytest.mark.parametrize("flexible", [False, True])
def test_traced_reference_model_runs_without_python_package(tmp_path, flexible):
    from torchff_b200.water import water_box_216

    wb = water_box_216()
    rng = np.random.default_rng(2)
    coords = (wb.coords + rng.normal(0.0, 0.004, wb.coords.shape)).astype(np.float32)
    model = Tip3pModel(wb, flexible).to("cuda")
    x = torch.tensor(coords, device="cuda", requires_grad=True)
    b = torch.tensor(wb.box, dtype=torch.float32, device="cuda")
    # eager through the drop-in modules, then traced as the reference traces Tip3pTorchFF
    e_eager = model(x, b)
    (g_eager,) = torch.autograd.grad(e_eager, x)
    traced = torch.jit.trace(model, (x.detach(), b), strict=False, check_trace=False)
    e = traced(x, b)
    (g,) = torch.autograd.grad(e, x)
    assert e.item() == e_eager.item() and torch.equal(g, g_eager)
    # the FP64 oracle on the same coordinates, at the mixed tolerances: energy within 1e-6 of
    # the summed term magnitudes, force RMS error below 1e-5
    orc = oracle_water(wb, coords.astype(np.float64), flexible=flexible)
    assert abs(e.item() - orc["energy"]) < 1e-6 * orc["scale"]
    assert rel_rms(g, orc["grad"]) < 1e-5
    # saved, then run by a process that loads only libtffb200_torch.so (what a C++ host does)
    p = tmp_path / "tip3p_traced.pt"
    traced.save(str(p))
    np.save(tmp_path / "x.npy", coords)
    np.save(tmp_path / "box.npy", np.asarray(wb.box, dtype=np.float32))
    code = textwrap.dedent(f"""
        import sys
        import numpy as np, torch
        torch.ops.load_library({_library_path()!r})
        m = torch.jit.load({str(p)!r})
        x = torch.tensor(np.load({str(tmp_path / 'x.npy')!r}), device="cuda", requires_grad=True)
        b = torch.tensor(np.load({str(tmp_path / 'box.npy')!r}), device="cuda")
        e = m(x, b)
        (g,) = torch.autograd.grad(e, x)
        np.save({str(tmp_path / 'g.npy')!r}, g.cpu().numpy())
        assert not any(k.startswith("torchff_b200") for k in sys.modules)
        print(repr(e.item()))
    """)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr[-2000:]
    assert float(r.stdout.strip().splitlines()[-1]) == e.item()
    assert np.array_equal(np.load(tmp_path / "g.npy"), g.cpu().numpy())
