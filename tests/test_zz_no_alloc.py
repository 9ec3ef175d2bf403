"""tff_nonbonded_atom_pairs_noalloc against tff_nonbonded_atom_pairs, both through the C ABI,
and against the reference's own values for the same inputs (golden pairs_random.npz).

The no-alloc entry point serves callers that may not allocate device memory (a force
plugin whose host MD engine owns all allocations, or a time-critical loop that must never
reach an allocator): it keeps its scratch in a static device array of libtffb200 instead
of a caller workspace. This file is collected last so a run that stops at the first
failure has run every other test; it also passes alone in a fresh process.

Tolerances are those of the pair-term tests: against the workspace entry point FP64
energies 1e-11 relative, gradients 1e-9 of their max magnitude, mixed precision 2e-6 and
1e-5; against the golden values FP64 1e-11 / 1e-9 and mixed 1e-5 / 1e-5 (rounding the FP64
inputs to FP32 bounds the mixed energies).
"""
import ctypes
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

TOL = {torch.float64: (1e-11, 1e-9), torch.float32: (2e-6, 1e-5)}
GOLDEN_TOL = {torch.float64: (1e-11, 1e-9), torch.float32: (1e-5, 1e-5)}


def _rel_max(a, b):
    a, b = a.double().cpu(), b.double().cpu()
    return float((a - b).abs().max() / b.abs().max().clamp_min(1e-300))


def _call(lib, fn, g, dtype, with_workspace):
    import torchff_b200._lib as L

    dev = torch.device("cuda")
    x = torch.tensor(g["coords"], dtype=dtype, device=dev)
    pairs = torch.tensor(g["pairs"], dtype=torch.int64, device=dev)
    box = torch.tensor(g["box"], dtype=dtype, device=dev)
    sig = torch.tensor(g["sigma"], dtype=dtype, device=dev)
    eps = torch.tensor(g["epsilon"], dtype=dtype, device=dev)
    q = torch.tensor(g["q"], dtype=dtype, device=dev)
    out = {"energy": torch.empty(1, dtype=dtype, device=dev), "gx": torch.empty_like(x),
           "gs": torch.empty_like(sig), "ge": torch.empty_like(eps), "gq": torch.empty_like(q)}
    args = [L.dtype_code(dtype), x.shape[0], L.ptr(x), pairs.shape[0], L.ptr(pairs), L.ptr(box), L.ptr(sig),
            L.ptr(eps), L.ptr(q), float(g["k"]), float(g["cutoff"]), 1, L.ptr(out["energy"]), L.ptr(out["gx"]),
            L.ptr(out["gs"]), L.ptr(out["ge"]), L.ptr(out["gq"])]
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    if with_workspace:
        ws = torch.empty(lib.tff_pairs_workspace_bytes(L.dtype_code(dtype), x.shape[0], 0), dtype=torch.uint8,
                         device=dev)
        st = fn(*args, L.ptr(ws), ws.numel(), stream)
    else:
        st = fn(*args, stream)
    assert st == 0, lib.tff_last_error().decode()
    torch.cuda.synchronize()
    return out


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_noalloc_matches_workspace_entry_point_twice(dtype):
    import torchff_b200._lib as L

    g = dict(np.load(os.path.join(GOLDEN, "pairs_random.npz")))
    lib = L.lib
    ref = _call(lib, lib.tff_nonbonded_atom_pairs, g, dtype, with_workspace=True)
    etol, gtol = TOL[dtype]
    getol, ggtol = GOLDEN_TOL[dtype]
    for _ in range(2):  # the shared static scratch must be cleared between calls
        got = _call(lib, lib.tff_nonbonded_atom_pairs_noalloc, g, dtype, with_workspace=False)
        assert abs(got["energy"].item() - ref["energy"].item()) <= etol * abs(ref["energy"].item())
        for k in ("gx", "gs", "ge", "gq"):
            assert _rel_max(got[k], ref[k]) < gtol, k
        # the reference's own result (shifted Coulomb + LJ with Lorentz-Berthelot combining)
        assert abs(got["energy"].item() - g["shift_energy"]) <= getol * abs(g["shift_energy"])
        for k in ("gx", "gs", "ge", "gq"):
            assert _rel_max(got[k], torch.tensor(g[f"shift_{k}"])) < ggtol, k


def test_noalloc_rejects_sizes_beyond_the_static_limit():
    import torchff_b200._lib as L

    lib = L.lib
    n = 65536 + 1
    st = lib.tff_nonbonded_atom_pairs_noalloc(L.TFF_F64, n, None, 0, None, None, None, None, None, 1.0, 1.0, 1,
                                              None, None, None, None, None, None)
    assert st == 1
    assert "limit" in lib.tff_last_error().decode()
