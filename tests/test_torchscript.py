"""TorchScript route for C++ hosts: the custom class in libtffb200_torch.so registers without a
GPU (CPU), and on the GPU a scripted, saved and reloaded model gives the energy and forces of
the Python path, also in a process that never imports torchff_b200."""
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest
import torch

from conftest import REPO
from gpu_util import oracle_water, rel_rms


def test_class_registers_and_pickles_without_gpu(tmp_path):
    from torchff_b200 import torchscript as TS
    from torchff_b200.water import water_box_216

    wb = water_box_216()
    m = torch.jit.script(TS.ScriptedTip3p(wb, flexible=True))
    assert m.system.natoms() == wb.natoms
    p = tmp_path / "tip3p.pt"
    torch.jit.save(m, str(p))
    m2 = torch.jit.load(str(p))
    assert m2.system.natoms() == wb.natoms


@pytest.mark.gpu
@pytest.mark.parametrize("flexible", [False, True])
def test_scripted_model_matches_python_path(tmp_path, flexible):
    from torchff_b200 import torchscript as TS
    from torchff_b200.system import FixedChargeSystem
    from torchff_b200.water import water_box_216

    wb = water_box_216()
    rng = np.random.default_rng(1)
    coords = wb.coords + rng.normal(0.0, 0.004, wb.coords.shape)
    x = torch.tensor(coords, dtype=torch.float32, device="cuda", requires_grad=True)
    b = torch.tensor(wb.box, dtype=torch.float32, device="cuda")
    m = torch.jit.script(TS.ScriptedTip3p(wb, flexible=flexible))
    e = m(x, b)
    (g,) = torch.autograd.grad(e, x)
    ref = FixedChargeSystem.from_water_box(wb, dtype=torch.float32, flexible=flexible).evaluate(x.detach(), b)
    # same library, same arithmetic: bit-identical energy and forces
    assert e.item() == np.float32(ref["energy"].item())
    assert torch.equal(-g, ref["forces"])
    # and the FP64 oracle on the same (FP32-rounded) coordinates, at the mixed tolerances:
    # energy within 1e-6 of the summed term magnitudes, force RMS error < 1e-5
    orc = oracle_water(wb, x.detach().double().cpu().numpy(), flexible=flexible)
    assert abs(e.item() - orc["energy"]) < 1e-6 * orc["scale"]
    assert rel_rms(-g, -orc["grad"]) < 1e-5
    e2, f2 = m.system.energy_forces(x.detach(), b)
    assert torch.equal(f2, ref["forces"])
    # saved, then run by a fresh process that only loads libtffb200_torch.so
    p = tmp_path / "tip3p.pt"
    torch.jit.save(m, str(p))
    np.save(tmp_path / "x.npy", coords)
    np.save(tmp_path / "box.npy", wb.box)
    code = textwrap.dedent(f"""
        import numpy as np, torch
        torch.ops.load_library({TS.library_path()!r})
        m = torch.jit.load({str(p)!r})
        x = torch.tensor(np.load({str(tmp_path / 'x.npy')!r}), dtype=torch.float32, device="cuda", requires_grad=True)
        b = torch.tensor(np.load({str(tmp_path / 'box.npy')!r}), dtype=torch.float32, device="cuda")
        e = m(x, b)
        (g,) = torch.autograd.grad(e, x)
        np.save({str(tmp_path / 'f.npy')!r}, (-g).cpu().numpy())
        print(repr(e.item()))
    """)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr[-2000:]
    assert "torchff_b200" not in r.stderr
    assert float(r.stdout.strip().splitlines()[-1]) == e.item()
    assert np.array_equal(np.load(tmp_path / "f.npy"), ref["forces"].cpu().numpy())
