"""Harmonic bonds and angles of flexible water: the operators against the golden fixture of
the reference's pure-torch HarmonicBond / HarmonicAngle / compute_angles_ref, and the fused
system with bonded terms against the oracle composition."""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from gpu_util import rel, rel_max, rel_rms, t
from oracle import oracle as O

pytestmark = pytest.mark.gpu

# FP64: 1e-12 relative (energies) / 1e-10 of the largest gradient component; FP32 inputs: 2e-6 / 2e-5
TOL = {torch.float64: (1e-12, 1e-10), torch.float32: (2e-6, 2e-5)}


def _golden():
    return np.load(os.path.join(GOLDEN, "bonded_water.npz"))


def _f32(a):
    return np.asarray(a).astype(np.float32).astype(np.float64)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_harmonic_bond_op(dtype):
    import torchff_b200  # noqa: F401
    from torchff_b200.bond import HarmonicBond, compute_harmonic_bond_forces

    g = _golden()
    x = t(g["coords"], dtype, True)
    b0, kb = t(g["b0"], dtype, True), t(g["kb"], dtype, True)
    bonds = torch.tensor(g["bonds"], device="cuda")
    e = HarmonicBond(use_customized_ops=True)(x, bonds, b0, kb)
    assert e.dim() == 0
    e.backward()
    cast = (lambda a: a) if dtype == torch.float64 else _f32
    E, gx, gb0, gk = O.harmonic_bond(cast(g["coords"]), g["bonds"], cast(g["b0"]), cast(g["kb"]))
    te, tg = TOL[dtype]
    assert rel(e.item(), E) < te
    assert rel_max(x.grad, gx) < tg and rel_max(b0.grad, gb0) < tg and rel_max(kb.grad, gk) < tg
    if dtype == torch.float64:  # against the reference's own autograd result
        assert rel(e.item(), float(g["bond_energy"])) < te and rel_max(x.grad, g["bond_gx"]) < tg
    f = torch.full_like(x.detach(), 2.0)
    compute_harmonic_bond_forces(x.detach(), bonds, b0.detach(), kb.detach(), f)
    assert rel_max(f - 2.0, -x.grad) < tg


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_harmonic_angle_op(dtype):
    import torchff_b200  # noqa: F401
    from torchff_b200.angle import HarmonicAngle, compute_harmonic_angle_forces

    g = _golden()
    x = t(g["coords"], dtype, True)
    th0, kth = t(g["th0"], dtype, True), t(g["kth"], dtype, True)
    ang = torch.tensor(g["angles"], device="cuda")
    e = HarmonicAngle(use_customized_ops=True)(x, ang, th0, kth)
    e.backward()
    cast = (lambda a: a) if dtype == torch.float64 else _f32
    E, gx, gt, gk = O.harmonic_angle(cast(g["coords"]), g["angles"], cast(g["th0"]), cast(g["kth"]))
    te, tg = TOL[dtype]
    if dtype == torch.float32:  # acos near the equilibrium angle amplifies FP32 rounding of cos
        te, tg = 2e-5, 1e-4
    assert rel(e.item(), E) < te
    assert rel_max(x.grad, gx) < tg and rel_max(th0.grad, gt) < tg and rel_max(kth.grad, gk) < tg
    if dtype == torch.float64:
        assert rel(e.item(), float(g["angle_energy"])) < te and rel_max(x.grad, g["angle_gx"]) < tg
    f = torch.zeros_like(x.detach())
    compute_harmonic_angle_forces(x.detach(), ang, th0.detach(), kth.detach(), f)
    assert rel_max(f, -x.grad) < tg


def test_compute_angles_and_backward():
    import torchff_b200  # noqa: F401
    from torchff_b200.angle import Angles

    g = _golden()
    x = t(g["coords"], grad=True)
    ang = torch.tensor(g["angles"], device="cuda")
    th = Angles(use_customized_ops=True)(x, ang)
    assert np.max(np.abs(th.detach().cpu().numpy() - g["theta"])) < 1e-13
    w = torch.linspace(0.5, 1.5, th.shape[0], dtype=torch.float64, device="cuda")
    (th * w).sum().backward()
    # d(sum w theta)/dx = the harmonic-angle gradient with k = 1 and theta - theta0 = w
    _, gx, _, _ = O.harmonic_angle(g["coords"], g["angles"], g["theta"] - w.cpu().numpy(), np.ones(th.shape[0]))
    assert rel_max(x.grad, gx) < 1e-10


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_flexible_system_vs_oracle(dtype):
    import torchff_b200  # noqa: F401
    from torchff_b200.system import FixedChargeSystem
    from torchff_b200.water import water_bonded_terms, water_box_216

    wb = water_box_216(seed=3)
    g = _golden()
    coords = g["coords"]  # distorted geometry of the same box
    sysm = FixedChargeSystem.from_water_box(wb, dtype=dtype, flexible=True)
    out = sysm.evaluate(t(coords, dtype), t(wb.box, dtype), terms=True)
    xo = coords if dtype == torch.float64 else _f32(coords)
    ref = O.fixed_charge_energy(xo, wb.box, wb.charges, wb.sigma_table, wb.epsilon_table, wb.atom_types,
                                wb.nblist_exclusions, wb.coulomb_exclusions, wb.cutoff, wb.alpha, wb.grid, 138.935456)
    bt = water_bonded_terms(wb.n_waters)
    eb, gb, _, _ = O.harmonic_bond(xo, bt.bonds, bt.b0, bt.kb)
    ea, ga, _, _ = O.harmonic_angle(xo, bt.angles, bt.th0, bt.kth)
    total = ref["total"] + eb + ea
    grad = ref["grad_coords"] + gb + ga
    terms = out["terms"].cpu().numpy()
    assert terms.shape == (6,)
    if dtype == torch.float64:
        assert rel(out["energy"].item(), total) < 1e-10
        assert rel(terms[4], eb) < 1e-12 and rel(terms[5], ea) < 1e-12
        assert rel_max(-out["forces"], grad) < 1e-8
    else:
        assert rel(terms[4], eb) < 2e-5 and rel(terms[5], ea) < 2e-5
        assert rel_rms(-out["forces"], grad) < 1e-5
    # the same forces through the first-derivative path; second derivatives are refused
    gr = sysm.evaluate_grads(t(coords, dtype), t(wb.box, dtype))
    assert rel_max(gr["forces"], out["forces"]) < (1e-12 if dtype == torch.float64 else 1e-6)
    with pytest.raises(RuntimeError, match="bonded"):
        sysm.hvp(t(coords, dtype), t(wb.box, dtype), t(np.ones_like(coords), dtype))
    # removing the bonded terms restores the nonbonded-only result
    sysm.set_bonded()
    out2 = sysm.evaluate(t(coords, dtype), t(wb.box, dtype))
    # the total is a near-cancelling sum: FP32 is held to 1e-6 of the summed component magnitudes
    scale = abs(ref["lj"]) + abs(ref["coul_real"]) + abs(138.935456 * ref["pme_raw"])
    err = abs(out2["energy"].item() - ref["total"])
    assert err < (1e-10 * abs(ref["total"]) if dtype == torch.float64 else 1e-6 * scale)


def test_flexible_host_path_matches_device_path():
    import torchff_b200  # noqa: F401
    from torchff_b200.system import FixedChargeSystem
    from torchff_b200.water import water_box_216

    wb = water_box_216(seed=3)
    coords = _golden()["coords"]
    sysm = FixedChargeSystem.from_water_box(wb, dtype=torch.float32, flexible=True)
    hf = np.zeros_like(coords)
    e_host = sysm.evaluate_host(np.ascontiguousarray(coords), np.ascontiguousarray(wb.box), hf)
    out = sysm.evaluate(t(coords, torch.float32), t(wb.box, torch.float32))
    assert e_host == out["energy"].item()
    assert np.array_equal(hf.astype(np.float32), out["forces"].cpu().numpy())
