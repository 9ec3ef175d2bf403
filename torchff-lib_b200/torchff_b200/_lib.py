"""ctypes binding of libtffb200.so (the C ABI declared in include/tffb200.h).

The library is the product: if it is missing or fails to load, importing this module
raises, and no operator falls back to another implementation.
"""
from __future__ import annotations

import ctypes as C
import os

import torch

from ._build import lib_path

TFF_F32, TFF_F64 = 0, 1
TFF_OK = 0
TFF_ERR_TIMEOUT = 6
_STATUS = {1: "invalid argument", 2: "CUDA error", 3: "cuFFT error", 4: "workspace too small",
           5: "capacity overflow", 6: "timeout"}

_path = lib_path()
if not os.path.exists(_path):
    raise ImportError(
        f"{_path} is not built; build it with `python -m torchff_b200._build` (nvcc, sm_100a)")
lib = C.CDLL(_path)

i32, i64, f64, vp, sz = C.c_int, C.c_int64, C.c_double, C.c_void_p, C.c_size_t


class SystemDesc(C.Structure):
    _fields_ = [("dtype", C.c_int), ("natoms", C.c_int64), ("cutoff", C.c_double),
                ("ewald_alpha", C.c_double), ("pme_grid", C.c_int), ("coul_constant", C.c_double),
                ("max_cluster_neighbors", C.c_int)]


class BatchDesc(C.Structure):
    _fields_ = [("dtype", C.c_int), ("max_systems", C.c_int), ("max_atoms", C.c_int64),
                ("max_grid_points", C.c_int64), ("cutoff", C.c_double), ("ewald_alpha", C.c_double),
                ("coul_constant", C.c_double), ("max_cluster_neighbors", C.c_int), ("atoms_per_cell", C.c_double)]


class ServerDesc(C.Structure):
    _fields_ = [("dtype", C.c_int), ("lanes", C.c_int), ("max_systems_per_batch", C.c_int),
                ("hbm_budget_bytes", C.c_size_t), ("grid_points_per_atom", C.c_double), ("cutoff", C.c_double),
                ("ewald_alpha", C.c_double), ("coul_constant", C.c_double), ("atoms_per_cell", C.c_double)]


class RequestDesc(C.Structure):
    _fields_ = [("natoms", C.c_int64), ("pme_grid", C.c_int), ("coords", C.c_void_p), ("box", C.c_void_p),
                ("charges", C.c_void_p), ("sigma", C.c_void_p), ("epsilon", C.c_void_p), ("nexcl", C.c_int64),
                ("excl_pairs", C.c_void_p), ("energy", C.c_void_p), ("forces", C.c_void_p)]


class ServerStats(C.Structure):
    _fields_ = [(name, C.c_int64) for name in (
        "submitted", "systems_launched", "systems_done", "batches", "max_batch_systems", "max_batch_atoms",
        "max_lanes_in_flight", "lane_max_atoms", "lane_max_grid_points", "lane_device_bytes")] + [("now", C.c_double)]


_SIGS = {
    "tff_version": (i32, []),
    "tff_last_error": (C.c_char_p, []),
    "tff_device_sm_count": (i32, []),
    "tff_nblist_nsquared": (i32, [i32, i64, vp, vp, f64, vp, vp, i32, vp, i64, vp, vp]),
    "tff_nblist_cell_list_workspace_bytes": (sz, [i32, i64, i32]),
    "tff_nblist_cell_list": (i32, [i32, i64, vp, vp, f64, vp, vp, i32, vp, i64, vp, i32, vp, sz, vp]),
    "tff_cluster_pairs_workspace_bytes": (sz, [i32, i64, i32]),
    "tff_cluster_pairs_build": (i32, [i32, i64, vp, vp, f64, vp, vp, vp, vp, vp, i64, vp, vp, i64, vp, i32, vp, sz,
                                      vp]),
    "tff_cluster_pairs_decode": (i32, [i32, i64, vp, vp, f64, vp, i64, vp, i64, vp, vp, vp, i64, vp, i64, vp, vp]),
    "tff_nonbonded_cluster_pairs_workspace_bytes": (sz, [i32, i64]),
    "tff_nonbonded_cluster_pairs": (i32, [i32, i64, vp, vp, vp, vp, vp, f64, f64, i32, vp, i64, vp, i64, vp, vp, vp,
                                          i64, vp, vp, vp, vp, vp, vp, vp, sz, vp]),
    "tff_nonbonded_forces_cluster_pairs": (i32, [i32, i64, vp, vp, vp, vp, vp, f64, f64, vp, i64, vp, i64, vp, vp,
                                                 vp, i64, vp, vp, sz, vp]),
    "tff_bonded_workspace_bytes": (sz, [i32, i64, i64]),
    "tff_harmonic_bond": (i32, [i32, i64, vp, i64, vp, vp, vp, vp, vp, vp, vp, vp, sz, vp]),
    "tff_harmonic_bond_forces": (i32, [i32, i64, vp, i64, vp, vp, vp, vp, vp, sz, vp]),
    "tff_harmonic_angle": (i32, [i32, i64, vp, i64, vp, vp, vp, vp, vp, vp, vp, vp, sz, vp]),
    "tff_harmonic_angle_forces": (i32, [i32, i64, vp, i64, vp, vp, vp, vp, vp, sz, vp]),
    "tff_angles": (i32, [i32, i64, vp, i64, vp, vp, vp, vp, vp, sz, vp]),
    "tff_pairs_workspace_bytes": (sz, [i32, i64, i64]),
    "tff_nonbonded_atom_pairs": (i32, [i32, i64, vp, i64, vp, vp, vp, vp, vp, f64, f64, i32, vp, vp, vp, vp, vp,
                                       vp, sz, vp]),
    "tff_nonbonded_atom_pairs_noalloc": (i32, [i32, i64, vp, i64, vp, vp, vp, vp, vp, f64, f64, i32, vp, vp, vp,
                                               vp, vp, vp]),
    "tff_nonbonded_forces_atom_pairs":(i32, [i32, i64, vp, i64, vp, vp, vp, vp, vp, f64, f64, vp, vp, sz, vp]),
    "tff_coulomb_atom_pairs": (i32, [i32, i64, vp, i64, vp, vp, vp, f64, f64, i32, vp, vp, vp, vp, sz, vp]),
    "tff_lennard_jones_atom_pairs": (i32, [i32, i64, vp, i64, vp, vp, vp, vp, f64, vp, i64, vp, vp, vp, vp, vp,
                                           sz, vp]),
    "tff_ewald_real_atom_pairs": (i32, [i32, i64, vp, vp, i64, vp, i64, vp, vp, f64, f64, f64, vp, vp, vp, vp,
                                        sz, vp]),
    "tff_pme_plan_create": (i32, [i32, i32, C.POINTER(vp)]),
    "tff_pme_plan_destroy": (i32, [vp]),
    "tff_pme_workspace_bytes": (sz, [vp, i64]),
    "tff_pme_long_range": (i32, [vp, i64, vp, vp, vp, f64, vp, vp, vp, vp, vp, vp, vp, sz, vp]),
    "tff_system_create": (i32, [C.POINTER(SystemDesc), vp, vp, vp, i64, vp, C.POINTER(vp)]),
    "tff_system_destroy": (i32, [vp]),
    "tff_system_set_bonded": (i32, [vp, i64, vp, vp, vp, i64, vp, vp, vp]),
    "tff_system_set_parameters": (i32, [vp, vp, vp, vp, vp]),
    "tff_system_eval": (i32, [vp, vp, vp, vp, vp, vp, vp, vp]),
    "tff_system_eval_host": (i32, [vp, vp, vp, vp, vp, vp]),
    "tff_system_status": (i32, [vp, vp, C.POINTER(C.c_int)]),
    "tff_timer_create": (i32, [C.POINTER(vp)]),
    "tff_timer_destroy": (i32, [vp]),
    "tff_timer_elapsed_ms": (i32, [vp, i32, i32, C.POINTER(C.c_float)]),
    "tff_system_eval_timed": (i32, [vp, vp, vp, vp, vp, vp, vp]),
    "tff_system_kernel_launches": (i32, [vp]),
    "tff_system_eval_grads": (i32, [vp, vp, vp, vp, vp, vp, vp, vp, vp]),
    "tff_system_hvp": (i32, [vp, vp, vp, vp, vp, vp, vp, vp, vp]),
    "tff_batch_device_bytes": (sz, [C.POINTER(BatchDesc)]),
    "tff_batch_create": (i32, [C.POINTER(BatchDesc), C.POINTER(vp)]),
    "tff_batch_destroy": (i32, [vp]),
    "tff_batch_eval": (i32, [vp, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
    "tff_batch_status": (i32, [vp, vp, C.POINTER(C.c_int)]),
    "tff_batch_kernel_launches": (i32, [vp]),
    "tff_batch_graph_launches": (C.c_int64, [vp]),
    "tff_server_create": (i32, [C.POINTER(ServerDesc), C.POINTER(vp)]),
    "tff_server_destroy": (i32, [vp]),
    "tff_server_submit": (i32, [vp, C.POINTER(RequestDesc), C.POINTER(i64)]),
    "tff_server_wait": (i32, [vp, i64, f64]),
    "tff_server_poll": (i32, [vp, i64, C.POINTER(C.c_int)]),
    "tff_server_request_times": (i32, [vp, i64, C.POINTER(f64), C.POINTER(f64), C.POINTER(f64)]),
    "tff_server_release": (i32, [vp, i64]),
    "tff_server_drain": (i32, [vp, f64]),
    "tff_server_get_stats": (i32, [vp, C.POINTER(ServerStats)]),
    "tff_server_hold": (i32, [vp, i32]),
}

for _name, (_res, _args) in _SIGS.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args

EXPORTED = tuple(_SIGS)


def check(status: int, what: str = "") -> None:
    if status != TFF_OK:
        msg = lib.tff_last_error().decode(errors="replace")
        raise RuntimeError(f"{what}: {_STATUS.get(status, status)}: {msg}")


def dtype_code(t: torch.dtype) -> int:
    if t == torch.float32:
        return TFF_F32
    if t == torch.float64:
        return TFF_F64
    raise TypeError(f"unsupported dtype {t}; expected float32 (mixed precision) or float64")


def ptr(t: torch.Tensor | None):
    return None if t is None else C.c_void_p(t.data_ptr())


def stream_of(t: torch.Tensor):
    return C.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def workspace(nbytes: int, device) -> torch.Tensor:
    return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)


def require_cuda(*tensors: torch.Tensor | None) -> None:
    for t in tensors:
        if t is not None and not t.is_cuda:
            raise RuntimeError("torchff_b200 operators need CUDA tensors")
