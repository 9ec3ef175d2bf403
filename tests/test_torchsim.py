"""torch-sim model interface (the reference's examples/tip3p/md_torchsim.py:98-140 wrapper):
units (Angstrom, eV, lattice vectors as cell columns) and the system layout checks on the
CPU; on the GPU one system against FixedChargeSystem and states of several uneven systems
(rigid and flexible water, FP64 and mixed) against each system evaluated alone.

Tolerances: the single-system path is the same evaluation on coordinates that went through
Angstrom and back (last-bit changes; 1e-12 in energy, 1e-11 of the largest force). A
batched system's reciprocal part is a direct DFT instead of cuFFT and its bonded terms come
from the bond / angle operators: against the same system alone in the same precision, FP64
agrees to 1e-10 relative in energy and 1e-9 of the largest force, mixed precision to 1e-8
of the summed energy-term magnitudes and 1e-6 of the largest force.
"""
from dataclasses import dataclass

import numpy as np
import pytest
import torch

from gpu_util import oracle_water, rel, rel_max


@dataclass
class FakeState:
    """The fields of torch-sim's SimState the model reads."""
    positions: torch.Tensor   # (N, 3) Angstrom
    cell: torch.Tensor        # (S, 3, 3) Angstrom, columns are lattice vectors
    system_idx: torch.Tensor  # (N,)

    @property
    def n_systems(self) -> int:
        return int(self.cell.shape[0])


def _state(boxes, device="cpu", order=None):
    pos = np.concatenate([wb.coords for wb in boxes]) * 10.0
    idx = np.concatenate([np.full(wb.natoms, k) for k, wb in enumerate(boxes)])
    if order is not None:
        pos, idx = pos[order], idx[order]
    cell = np.stack([wb.box.T * 10.0 for wb in boxes])
    return FakeState(torch.tensor(pos, dtype=torch.float64, device=device),
                     torch.tensor(cell, dtype=torch.float64, device=device), torch.tensor(idx, device=device))


def test_units_layout_and_interface_without_gpu():
    from torchff_b200 import torchsim as TS
    from torchff_b200.water import serving_water_box

    boxes = [serving_water_box(n, seed=k) for k, n in enumerate((64, 150))]
    st = _state(boxes)
    nm = TS.boxes_nm(st.cell)
    for k, wb in enumerate(boxes):
        assert np.allclose(nm[k].numpy(), wb.box, rtol=0, atol=1e-15)
    off = TS.system_offsets(st.system_idx, [wb.natoms for wb in boxes])
    assert off.tolist() == [0, boxes[0].natoms, boxes[0].natoms + boxes[1].natoms]
    with pytest.raises(ValueError):
        TS.system_offsets(st.system_idx.flip(0), [wb.natoms for wb in boxes])
    with pytest.raises(ValueError):
        TS.system_offsets(st.system_idx, [boxes[0].natoms + 3, boxes[1].natoms - 3])
    tops = [TS.Topology.from_water_box(wb, flexible=True) for wb in boxes]
    m = TS.TorchSimModel(tops, 0.9, boxes[0].alpha)
    assert m.compute_forces and not m.compute_stress and m.dtype == torch.float64
    assert m.memory_scales_with == "n_atoms" and m.device.type == "cuda"
    with pytest.raises(NotImplementedError):
        TS.TorchSimModel(tops, 0.9, boxes[0].alpha, compute_stress=True)


@pytest.mark.gpu
@pytest.mark.parametrize("flexible", [False, True])
def test_single_system_matches_fixed_charge_system(flexible):
    from torchff_b200 import torchsim as TS
    from torchff_b200.system import FixedChargeSystem
    from torchff_b200.water import water_box_216

    wb = water_box_216()
    m = TS.TorchSimModel(TS.Topology.from_water_box(wb, flexible=flexible), wb.cutoff, wb.alpha,
                         compute_dtype=torch.float64)
    out = m(_state([wb], "cuda"))
    ref = FixedChargeSystem.from_water_box(wb, dtype=torch.float64, flexible=flexible).evaluate(
        torch.tensor(wb.coords, device="cuda"), torch.tensor(wb.box, device="cuda"))
    assert out["energy"].shape == (1,) and out["forces"].shape == (wb.natoms, 3)
    assert rel(out["energy"][0] * TS.KJMOL_PER_EV, ref["energy"]) < 1e-12
    assert rel_max(out["forces"] * (TS.KJMOL_PER_EV / TS.NM_PER_ANGSTROM), ref["forces"]) < 1e-11
    # the FP64 oracle in the reference's units: energy 1e-10 relative, forces 1e-8 of the largest
    orc = oracle_water(wb, flexible=flexible)
    assert rel(out["energy"][0] * TS.KJMOL_PER_EV, orc["energy"]) < 1e-10
    assert rel_max(out["forces"] * (TS.KJMOL_PER_EV / TS.NM_PER_ANGSTROM), -orc["grad"]) < 1e-8


@pytest.mark.gpu
@pytest.mark.parametrize("compute_dtype", [torch.float64, torch.float32])
def test_several_systems_match_each_system_alone(compute_dtype):
    from torchff_b200 import torchsim as TS
    from torchff_b200.system import FixedChargeSystem
    from torchff_b200.water import serving_water_box

    boxes = [serving_water_box(n, seed=10 + k) for k, n in enumerate((150, 700, 333))]
    flex = [True, False, True]
    tops = [TS.Topology.from_water_box(wb, flexible=f) for wb, f in zip(boxes, flex)]
    m = TS.TorchSimModel(tops, 0.9, boxes[0].alpha, compute_dtype=compute_dtype)
    st = _state(boxes, "cuda")
    out = m(st)
    assert out["energy"].shape == (3,) and out["forces"].dtype == torch.float64
    off = np.concatenate([[0], np.cumsum([wb.natoms for wb in boxes])])
    for k, (wb, f) in enumerate(zip(boxes, flex)):
        x = torch.tensor(np.asarray(st.positions[off[k]:off[k + 1]].cpu()) * TS.NM_PER_ANGSTROM, device="cuda")
        ref = FixedChargeSystem.from_water_box(wb, dtype=compute_dtype, flexible=f).evaluate(
            x.to(compute_dtype), torch.tensor(wb.box, dtype=compute_dtype, device="cuda"), terms=True)
        e = float(out["energy"][k]) * TS.KJMOL_PER_EV
        fk = out["forces"][off[k]:off[k + 1]] * (TS.KJMOL_PER_EV / TS.NM_PER_ANGSTROM)
        if compute_dtype == torch.float64:
            assert rel(e, ref["energy"]) < 1e-10
            assert rel_max(fk, ref["forces"]) < 1e-9
        else:
            assert abs(e - float(ref["energy"])) < 1e-8 * float(ref["terms"].abs().sum())
            assert rel_max(fk, ref["forces"]) < 1e-6
    # a second step with moved atoms reuses the packed parameters
    st.positions += 0.01
    out2 = m(st)
    assert not torch.equal(out2["forces"], out["forces"])


@pytest.mark.gpu
def test_atoms_out_of_system_order_are_refused():
    from torchff_b200 import torchsim as TS
    from torchff_b200.water import serving_water_box

    boxes = [serving_water_box(n, seed=k) for k, n in enumerate((100, 120))]
    m = TS.TorchSimModel([TS.Topology.from_water_box(wb) for wb in boxes], 0.9, boxes[0].alpha)
    n = sum(wb.natoms for wb in boxes)
    with pytest.raises(ValueError):
        m(_state(boxes, "cuda", order=np.random.default_rng(0).permutation(n)))
