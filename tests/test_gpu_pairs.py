"""Pair-term operators vs the golden fixtures (reference pure-torch outputs) and the oracle.

Tolerances: FP64 energies 1e-11 relative, gradients 1e-9 of their max magnitude;
mixed precision (FP32 inputs) energies 1e-5 relative, gradients 1e-5 of max magnitude.
The FP32 energy bound is set by rounding the FP64 golden inputs to FP32 (about 1e-7
per distance) inside near-cancelling sums, not by the kernel arithmetic.
"""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from gpu_util import rel, rel_max, t
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = {torch.float64: (1e-11, 1e-9), torch.float32: (1e-5, 1e-5)}
DTYPES = [torch.float64, torch.float32]


@pytest.fixture(scope="module")
def g():
    import torchff_b200  # noqa: F401

    return dict(np.load(os.path.join(GOLDEN, "pairs_random.npz")))


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("tag,shift", [("shift", True), ("noshift", False)])
def test_nonbonded_op(g, dtype, tag, shift):
    x, q, s, e = (t(g[k], dtype, grad=True) for k in ("coords", "q", "sigma", "epsilon"))
    ene = torch.ops.torchff.compute_nonbonded_energy_from_atom_pairs(
        x, t(g["pairs"], torch.int64), t(g["box"], dtype), s, e, q, float(g["k"]), float(g["cutoff"]), shift)
    assert ene.shape == (1,) and ene.dtype == dtype
    ene.sum().backward()
    et, gt = TOL[dtype]
    assert rel(ene.item(), g[f"{tag}_energy"]) < et
    for a, b in ((x.grad, "gx"), (q.grad, "gq"), (s.grad, "gs"), (e.grad, "ge")):
        assert rel_max(a, g[f"{tag}_{b}"]) < gt, b


@pytest.mark.parametrize("dtype", DTYPES)
def test_nonbonded_forces_op_adds(g, dtype):
    x = t(g["coords"], dtype)
    f = torch.ones_like(x)
    torch.ops.torchff.compute_nonbonded_forces_from_atom_pairs(
        x, t(g["pairs"], torch.int64), t(g["box"], dtype), t(g["sigma"], dtype), t(g["epsilon"], dtype),
        t(g["q"], dtype), float(g["k"]), float(g["cutoff"]), f)
    assert rel_max(f - 1.0, -g["shift_gx"]) < TOL[dtype][1]


@pytest.mark.parametrize("dtype", DTYPES)
def test_coulomb_op(g, dtype):
    x, q = t(g["coords"], dtype, grad=True), t(g["q"], dtype, grad=True)
    ene = torch.ops.torchff.compute_coulomb_energy(x, t(g["pairs"], torch.int64), t(g["box"], dtype), q,
                                                   float(g["k"]), float(g["cutoff"]), True)
    ene.sum().backward()
    e0, gx0, gq0 = O.coulomb(g["coords"], g["pairs"], g["box"], g["q"], float(g["k"]), float(g["cutoff"]), True)
    assert rel(ene.item(), g["shift_coul"]) < TOL[dtype][0] and rel(e0, g["shift_coul"]) < 1e-13
    assert rel_max(x.grad, gx0) < TOL[dtype][1] and rel_max(q.grad, gq0) < TOL[dtype][1]


@pytest.mark.parametrize("dtype", DTYPES)
def test_lj_per_pair(g, dtype):
    x = t(g["coords"], dtype, grad=True)
    s, e = t(g["lj_pair_sigma"], dtype, grad=True), t(g["lj_pair_epsilon"], dtype, grad=True)
    ene = torch.ops.torchff.compute_lennard_jones_energy(x, t(g["pairs"], torch.int64), t(g["box"], dtype), s, e,
                                                         float(g["cutoff"]), None)
    assert ene.dim() == 0
    ene.backward()
    assert rel(ene.item(), g["lj_pair_energy"]) < TOL[dtype][0]
    for a, b in ((x.grad, "lj_pair_gx"), (s.grad, "lj_pair_gs"), (e.grad, "lj_pair_ge")):
        assert rel_max(a, g[b]) < TOL[dtype][1], b


@pytest.mark.parametrize("dtype", DTYPES)
def test_lj_type_tables(g, dtype):
    from torchff_b200.vdw import Vdw

    x = t(g["coords"], dtype, grad=True)
    s, e = t(g["lj_type_sigma"], dtype, grad=True), t(g["lj_type_epsilon"], dtype, grad=True)
    vdw = Vdw("LennardJones", use_customized_ops=True, use_type_pairs=True)
    ene = vdw(x, t(g["pairs"], torch.int64), t(g["box"], dtype), s, e, float(g["cutoff"]),
              atom_types=t(g["lj_type_types"], torch.int64))
    ene.backward()
    assert rel(ene.item(), g["lj_type_energy"]) < TOL[dtype][0]
    for a, b in ((x.grad, "lj_type_gx"), (s.grad, "lj_type_gs"), (e.grad, "lj_type_ge")):
        assert rel_max(a, g[b]) < TOL[dtype][1], b


@pytest.mark.parametrize("dtype", DTYPES)
def test_ewald_real_with_exclusions(g, dtype):
    from torchff_b200.multipoles import MultipolarInteraction

    x, q = t(g["coords"], dtype, grad=True), t(g["q"], dtype, grad=True)
    mi = MultipolarInteraction(0, float(g["cutoff"]), float(g["ewald_alpha"]), 138.935456)
    ene = mi(x, t(g["box"], dtype), t(g["ewald_pairs"], torch.int64), q,
             pairs_excl=t(g["ewald_excl"], torch.int64))
    assert ene.dim() == 0
    ene.backward()
    assert rel(ene.item(), g["ewald_energy"]) < TOL[dtype][0] * 10
    assert rel_max(x.grad, g["ewald_gx"]) < TOL[dtype][1] and rel_max(q.grad, g["ewald_gq"]) < TOL[dtype][1]


def test_plain_coulomb_when_alpha_negative(g):
    x = t(g["coords"], grad=True)
    q = t(g["q"])
    ene = torch.ops.torchff.compute_multipolar_energy_from_atom_pairs(
        x, t(g["box"]), t(g["ewald_pairs"], torch.int64), t(g["ewald_excl"], torch.int64), q, None, None,
        float(g["cutoff"]), -1.0, 2.0)
    e0, gx0, _ = O.ewald_real(g["coords"], g["box"], g["ewald_pairs"], g["q"], float(g["cutoff"]), -1.0, 2.0,
                              g["ewald_excl"])
    ene.backward()
    assert rel(ene.item(), e0) < 1e-11 and rel_max(x.grad, gx0) < 1e-9


def test_mixed_precision_gradients_are_bit_reproducible(g):
    outs = []
    for _ in range(3):
        x, q, s, e = (t(g[k], torch.float32, grad=True) for k in ("coords", "q", "sigma", "epsilon"))
        ene = torch.ops.torchff.compute_nonbonded_energy_from_atom_pairs(
            x, t(g["pairs"], torch.int64), t(g["box"], torch.float32), s, e, q, 138.935456, 0.5, True)
        ene.sum().backward()
        outs.append([ene.detach().cpu()] + [v.grad.cpu() for v in (x, q, s, e)])
    for o in outs[1:]:
        for a, b in zip(o, outs[0]):
            assert torch.equal(a, b)


def test_rank_above_zero_raises(g):
    with pytest.raises(Exception):
        torch.ops.torchff.compute_multipolar_energy_from_atom_pairs(
            t(g["coords"]), t(g["box"]), t(g["pairs"], torch.int64), None, t(g["q"]), t(g["coords"]), None,
            0.5, 3.0, 1.0)


def test_padding_rows_are_skipped(g):
    pairs = np.concatenate([g["pairs"], -np.ones((50, 2), np.int64)], 0)
    ene = torch.ops.torchff.compute_coulomb_energy(t(g["coords"]), t(pairs, torch.int64), t(g["box"]), t(g["q"]),
                                                   float(g["k"]), float(g["cutoff"]), True)
    assert rel(ene.item(), g["shift_coul"]) < 1e-11


def test_empty_pair_list(g):
    ene = torch.ops.torchff.compute_coulomb_energy(t(g["coords"]), torch.zeros((0, 2), dtype=torch.int64,
                                                   device="cuda"), t(g["box"]), t(g["q"]), 1.0, 0.5, True)
    assert ene.item() == 0.0
