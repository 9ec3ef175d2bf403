"""The ctypes binding a Python maintainer adds to call libtffb200's C ABI directly.

This is the minimal stub for one entry point, tff_nonbonded_atom_pairs (the kernel behind
torch.ops.torchff.compute_nonbonded_energy_from_atom_pairs,
csrc/nonbonded/nonbonded_interface.cpp:9 in the reference), written the way a caller
outside this package would write it; ``torchff_b200/_lib.py`` holds the full table for
every symbol. A CPU test checks these declarations against ``include/tffb200.h``.

    import torch
    from torchff_b200.capi_example import load, nonbonded_energy
    lib = load()
    e = nonbonded_energy(lib, x, pairs, box, sigma, epsilon, q, cutoff=1.0)
"""
from __future__ import annotations

import ctypes as C
import os

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libtffb200.so")


def load(path: str = LIB_PATH) -> C.CDLL:
    lib = C.CDLL(path)
    lib.tff_pairs_workspace_bytes.restype = C.c_size_t
    lib.tff_pairs_workspace_bytes.argtypes = [C.c_int, C.c_int64, C.c_int64]
    lib.tff_last_error.restype = C.c_char_p
    lib.tff_last_error.argtypes = []
    lib.tff_nonbonded_atom_pairs.restype = C.c_int
    lib.tff_nonbonded_atom_pairs.argtypes = [
        C.c_int, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p,   # dtype, N, coords, P, pairs, box
        C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_int,  # sigma, eps, q, k, cutoff, shift
        C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,           # energy, dE/dx, dE/dsigma, dE/deps, dE/dq
        C.c_void_p, C.c_size_t, C.c_void_p]                                   # workspace, its bytes, stream
    return lib


def nonbonded_energy(lib: C.CDLL, x, pairs, box, sigma, epsilon, q, cutoff: float, coul_constant: float = 138.935456,
                     do_shift: bool = True):
    """Energy (1,) and dE/dx (N,3) of the shifted Coulomb + LJ pair term, on torch's current
    stream; float32 or float64 CUDA tensors, pairs (P,2) int64."""
    import torch

    dtype_code = {torch.float32: 0, torch.float64: 1}[x.dtype]
    n, p = x.shape[0], pairs.shape[0]
    energy = torch.empty(1, dtype=x.dtype, device=x.device)
    gx = torch.empty_like(x)
    ws = torch.empty(lib.tff_pairs_workspace_bytes(dtype_code, n, 0), dtype=torch.uint8, device=x.device)
    st = lib.tff_nonbonded_atom_pairs(dtype_code, n, x.data_ptr(), p, pairs.data_ptr(), box.data_ptr(),
                                      sigma.data_ptr(), epsilon.data_ptr(), q.data_ptr(), coul_constant, cutoff,
                                      int(do_shift), energy.data_ptr(), gx.data_ptr(), None, None, None,
                                      ws.data_ptr(), ws.numel(), torch.cuda.current_stream(x.device).cuda_stream)
    if st != 0:
        raise RuntimeError(f"tff_nonbonded_atom_pairs failed ({st}): {lib.tff_last_error().decode()}")
    return energy, gx
