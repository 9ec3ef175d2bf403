"""PME (rank 0) vs the reference's pure-torch outputs and the oracle."""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from gpu_util import rel, rel_max, rel_rms, t
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype,etol,gtol", [(torch.float64, 1e-11, 1e-9), (torch.float32, 2e-6, 2e-5)])
def test_reference_input_300(dtype, etol, gtol):
    from torchff_b200.pme import PME

    g = np.load(os.path.join(GOLDEN, "pme_random300.npz"))
    pme = PME(float(g["alpha"]), int(g["K"]), 0, use_customized_ops=True).cuda()
    x, q = t(g["coords"], dtype, grad=True), t(g["q"], dtype, grad=True)
    e = pme(x, t(g["box"], dtype), q)
    assert e.dim() == 0 and e.dtype == dtype
    e.backward()
    assert rel(e.item(), g["energy"]) < etol
    assert rel_max(x.grad, g["gx"]) < gtol and rel_max(q.grad, g["gq"]) < gtol


@pytest.mark.parametrize("dtype,etol,gtol", [(torch.float64, 1e-11, 1e-9), (torch.float32, 2e-6, 2e-5)])
def test_water216(dtype, etol, gtol):
    from torchff_b200.pme import PME

    g = np.load(os.path.join(GOLDEN, "water216.npz"))
    pme = PME(float(g["alpha"]), int(g["grid"]), 0, use_customized_ops=True).cuda()
    x, q = t(g["coords"], dtype, grad=True), t(g["charges"], dtype, grad=True)
    e = pme(x, t(g["box"], dtype), q)
    e.backward()
    assert rel(e.item(), g["e_pme"]) < etol
    assert rel_max(x.grad, g["gx_pme"]) < gtol and rel_max(q.grad, g["gq_pme"]) < gtol


@pytest.mark.parametrize("K", [13, 21, 32])
def test_odd_and_even_grids_triclinic(K):
    from torchff_b200.pme import PME

    rng = np.random.default_rng(K)
    box = np.array([[2.4, 0.0, 0.0], [0.3, 2.2, 0.0], [-0.2, 0.4, 2.5]])
    x = rng.random((400, 3)) @ box
    q = rng.standard_normal(400)
    q -= q.mean()
    e0, gx0, pot0, _ = O.pme(x, box, q, 3.1, K)
    pme = PME(3.1, K, 0, use_customized_ops=True).cuda()
    xt, qt = t(x, grad=True), t(q, grad=True)
    e = pme(xt, t(box), qt)
    e.backward()
    assert rel(e.item(), e0) < 1e-11
    assert rel_max(xt.grad, gx0) < 1e-9 and rel_max(qt.grad, pot0) < 1e-9


def test_mixed_precision_is_deterministic_and_accurate():
    from torchff_b200.pme import PME
    from torchff_b200.water import water_box_3000

    wb = water_box_3000()
    e0, gx0, pot0, _ = O.pme(wb.coords, wb.box, wb.charges, wb.alpha, wb.grid)
    pme = PME(wb.alpha, wb.grid, 0, use_customized_ops=True).cuda()
    res = []
    for _ in range(2):
        x = t(wb.coords, torch.float32, grad=True)
        e = pme(x, t(wb.box, torch.float32), t(wb.charges, torch.float32))
        e.backward()
        res.append((e.detach().cpu(), x.grad.cpu()))
    assert torch.equal(res[0][0], res[1][0]) and torch.equal(res[0][1], res[1][1])
    assert rel(res[0][0].item(), e0) < 2e-6
    assert rel_rms(res[0][1], gx0) < 1e-5


def test_mixed_spread_grid_does_not_depend_on_atom_order():
    """The FP32 spread sums each group of three consecutive atoms (a water here) over the
    union window of their stencils, and spreads atoms whose group is too spread out one by
    one; either way every contribution is rounded to fixed point alone and the integers are
    summed. A random permutation of the atoms breaks the groups apart (other code paths, other
    atomics), yet the grid, and so the energy and the forces, must be bit-identical."""
    from torchff_b200.pme import PME
    from torchff_b200.water import water_box_3000

    wb = water_box_3000()
    perm = np.random.default_rng(5).permutation(wb.natoms)
    inv = np.argsort(perm)
    pme = PME(wb.alpha, wb.grid, 0, use_customized_ops=True).cuda()
    out = []
    for order in (np.arange(wb.natoms), perm):
        x = t(wb.coords[order], torch.float32, grad=True)
        q = t(wb.charges[order], torch.float32, grad=True)
        e = pme(x, t(wb.box, torch.float32), q)
        e.backward()
        out.append((e.detach().cpu(), x.grad.cpu(), q.grad.cpu()))
    back = torch.as_tensor(inv)
    assert torch.equal(out[0][0], out[1][0])
    assert torch.equal(out[0][1], out[1][1][back])
    assert torch.equal(out[0][2], out[1][2][back])
