"""First and second derivatives of the fused system (force matching).

FP64 against the torch float64 oracle (autograd, including the double backward of a
force-matching loss) on 216 waters: 1e-8 of the largest component for first derivatives,
1e-7 for second derivatives. Central finite differences (step 1e-6, FP64) of the same loss
with respect to charges, sigma and epsilon agree with the double-backward gradient to 1e-5
relative. dE/deps_i is 0 where eps_i = 0 (TIP3P hydrogens), in the CUDA path and the oracle.
Mixed precision second derivatives agree with FP64 to 1e-4 (RMS relative).
"""
import numpy as np
import pytest
import torch

from gpu_util import rel, rel_max, rel_rms
from oracle import oracle as O
from oracle import torch_energy as TE

pytestmark = pytest.mark.gpu


def _setup(wb, seed, all_lj=False):
    from torchff_b200.water import force_matching_parameters

    q, s, e = force_matching_parameters(wb, seed)
    if all_lj:  # every atom with LJ (exercises sigma/epsilon paths of all atom pairs)
        h = wb.atom_types == 1
        s[h], e[h] = 0.1, 0.02
    rng = np.random.default_rng(seed + 1)
    target = rng.normal(0.0, 300.0, size=wb.coords.shape)
    return q, s, e, target


def _ours(wb, q, s, e, target, dtype=torch.float64, coords=None):
    from torchff_b200.system import FixedChargeNonbonded, FixedChargeSystem

    sysm = FixedChargeSystem(q, s, e, wb.coulomb_exclusions, wb.cutoff, wb.alpha, wb.grid, dtype=dtype)
    model = FixedChargeNonbonded(sysm)
    c = wb.coords if coords is None else coords
    x = torch.tensor(c, dtype=dtype, device="cuda", requires_grad=True)
    box = torch.tensor(wb.box, dtype=dtype, device="cuda")
    qq, ss, ee = (torch.tensor(a, dtype=dtype, device="cuda", requires_grad=True) for a in (q, s, e))
    E = model(x, box, qq, ss, ee)
    gx, gq, gs, ge = torch.autograd.grad(E, (x, qq, ss, ee), create_graph=True)
    F = -gx
    loss = torch.mean((F - torch.tensor(target, dtype=dtype, device="cuda")) ** 2)
    loss.backward()
    return {"E": E.item(), "F": F.detach(), "gq": gq.detach(), "gs": gs.detach(), "ge": ge.detach(),
            "loss": loss.item(), "dq": qq.grad, "ds": ss.grad, "de": ee.grad, "dx": x.grad, "system": sysm}


def _oracle(wb, q, s, e, target):
    rp, col = O.exclusions_coo_to_csr(wb.nblist_exclusions, wb.natoms)
    pairs = torch.tensor(O.nblist_pairs(wb.coords, wb.box, wb.cutoff, rp, col))
    x = torch.tensor(wb.coords, requires_grad=True)
    qq, ss, ee = (torch.tensor(a, requires_grad=True) for a in (q, s, e))
    E = TE.fixed_charge_energy(x, torch.tensor(wb.box), qq, ss, ee, pairs, torch.tensor(wb.coulomb_exclusions),
                               wb.cutoff, wb.alpha, wb.grid)
    gx, gq, gs, ge = torch.autograd.grad(E, (x, qq, ss, ee), create_graph=True)
    loss = torch.mean((-gx - torch.tensor(target)) ** 2)
    loss.backward()
    return {"E": E.item(), "F": -gx.detach(), "gq": gq.detach(), "gs": gs.detach(), "ge": ge.detach(),
            "loss": loss.item(), "dq": qq.grad, "ds": ss.grad, "de": ee.grad, "dx": x.grad}


@pytest.mark.parametrize("all_lj", [False, True])
def test_first_and_second_derivatives_match_torch_oracle(all_lj):
    from torchff_b200.water import water_box_216

    wb = water_box_216()
    q, s, e, target = _setup(wb, 3, all_lj)
    ours = _ours(wb, q, s, e, target)
    ref = _oracle(wb, q, s, e, target)
    assert rel(ours["E"], ref["E"]) < 1e-10
    for k in ("F", "gq", "gs", "ge"):
        assert rel_max(ours[k], ref[k]) < 1e-8, k
    assert rel(ours["loss"], ref["loss"]) < 1e-10
    for k in ("dq", "ds", "de", "dx"):
        assert rel_max(ours[k], ref[k]) < 1e-7, k
    if not all_lj:
        h = wb.atom_types == 1
        assert torch.all(ours["ge"][torch.tensor(h, device="cuda")] == 0)


def test_force_matching_gradient_matches_finite_differences():
    """3000 waters, FP64: central differences of the loss (step 1e-6) on charges of an O and
    an H atom and on sigma and epsilon of two O atoms."""
    from torchff_b200.water import water_box_3000

    wb = water_box_3000()
    q, s, e, target = _setup(wb, 7)
    ours = _ours(wb, q, s, e, target)
    sysm = ours["system"]
    x = torch.tensor(wb.coords, dtype=torch.float64, device="cuda")
    box = torch.tensor(wb.box, dtype=torch.float64, device="cuda")
    tt = torch.tensor(target, dtype=torch.float64, device="cuda")

    def loss(qv, sv, ev):
        sysm.set_parameters(*(torch.tensor(a, dtype=torch.float64, device="cuda") for a in (qv, sv, ev)))
        F = sysm.evaluate(x, box)["forces"]
        return float(torch.mean((F - tt) ** 2))

    h = 1e-6
    checks = [("dq", 0, 30), ("dq", 0, 31), ("ds", 1, 60), ("ds", 1, 903), ("de", 2, 60), ("de", 2, 903)]
    for name, which, atom in checks:
        plus = [q.copy(), s.copy(), e.copy()]
        minus = [q.copy(), s.copy(), e.copy()]
        plus[which][atom] += h
        minus[which][atom] -= h
        fd = (loss(*plus) - loss(*minus)) / (2 * h)
        g = float(ours[name][atom])
        assert abs(fd - g) <= 1e-5 * max(abs(g), 1e-3 * float(ours[name].abs().max())), (name, atom, fd, g)


def test_mixed_precision_second_derivatives_track_fp64():
    from torchff_b200.water import water_box_216

    wb = water_box_216()
    q, s, e, target = _setup(wb, 11)
    d64 = _ours(wb, q, s, e, target, torch.float64)
    d32 = _ours(wb, q, s, e, target, torch.float32)
    for k in ("dq", "ds", "dx"):
        assert rel_rms(d32[k], d64[k]) < 1e-4, k
