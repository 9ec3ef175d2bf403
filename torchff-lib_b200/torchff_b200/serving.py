"""Many periodic systems per launch: the batched evaluator and the continuous-batching server.

The reference evaluates one system per call (its torch-sim wrapper,
examples/tip3p/md_torchsim.py:113-140, rejects ``n_systems != 1``); this module has no
reference counterpart. Physics and precision are those of :class:`FixedChargeSystem`
(fused LJ + erfc Coulomb with Ewald exclusion correction + rank-0 PME, order 6), and a
system's result does not depend on what else is evaluated with it.

* :class:`BatchEvaluator` -- ``tff_batch``: a list of systems (device arrays) evaluated
  by one launch per stage.
* :class:`Server` -- ``tff_server``: requests (host arrays) are queued; a native worker
  thread keeps several batches ("lanes") in flight on their own streams and starts every
  free lane with as many queued requests as fit its share of the HBM budget.
* :func:`autotune_atoms_per_cell` -- picks the cell-grid occupancy that evaluates a sample
  batch fastest.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import check, lib

EXCL_SLOTS = 8
MAX_ATOMS_PER_SYSTEM = 16384


@dataclass
class SystemSpec:
    """One periodic system: host float64 arrays and system-local exclusion pairs."""
    coords: np.ndarray      # (n, 3)
    box: np.ndarray         # (3, 3), rows are box vectors
    charges: np.ndarray     # (n,)
    sigma: np.ndarray       # (n,)
    epsilon: np.ndarray     # (n,)
    excl_pairs: np.ndarray  # (m, 2) int64
    pme_grid: int

    @property
    def natoms(self) -> int:
        return int(self.coords.shape[0])

    @classmethod
    def from_water_box(cls, wb) -> "SystemSpec":
        return cls(np.ascontiguousarray(wb.coords, dtype=np.float64), np.ascontiguousarray(wb.box, dtype=np.float64),
                   np.ascontiguousarray(wb.charges, dtype=np.float64), np.ascontiguousarray(wb.sigma, dtype=np.float64),
                   np.ascontiguousarray(wb.epsilon, dtype=np.float64),
                   np.ascontiguousarray(wb.coulomb_exclusions, dtype=np.int64), int(wb.grid))


def exclusion_table(natoms: int, pairs: np.ndarray) -> np.ndarray:
    """(natoms, 8) int32 excluded partners per atom (both directions, self dropped,
    deduplicated, ascending), -1 padded; the layout tff_batch_eval takes."""
    p = np.asarray(pairs, dtype=np.int64).reshape(-1, 2)
    p = p[p[:, 0] != p[:, 1]]
    both = np.unique(np.concatenate([p, p[:, ::-1]]), axis=0)
    out = np.full((natoms, EXCL_SLOTS), -1, dtype=np.int32)
    if both.size == 0:
        return out
    rows, cols = both[:, 0], both[:, 1]
    start = np.searchsorted(rows, rows, side="left")
    rank = np.arange(rows.size) - start
    if rank.max() >= EXCL_SLOTS:
        raise ValueError(f"an atom has more than {EXCL_SLOTS} excluded partners")
    out[rows, rank] = cols
    return out


class BatchEvaluator:
    """Evaluates lists of systems with one launch per stage (``tff_batch``)."""

    def __init__(self, cutoff: float, ewald_alpha: float, dtype: torch.dtype = torch.float32,
                 max_systems: int = 256, max_atoms: int = 1 << 20, max_grid_points: int = 1 << 24,
                 coul_constant: float = 138.935456, atoms_per_cell: float = 0.0, device=None):
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.dtype = dtype
        self.desc = _lib.BatchDesc(_lib.dtype_code(dtype), int(max_systems), int(max_atoms), int(max_grid_points),
                                   float(cutoff), float(ewald_alpha), float(coul_constant), 0, float(atoms_per_cell))
        self._h = C.c_void_p()
        with torch.cuda.device(self.device):
            check(lib.tff_batch_create(C.byref(self.desc), C.byref(self._h)), "tff_batch_create")

    def close(self) -> None:
        if self._h:
            lib.tff_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def device_bytes(self) -> int:
        return int(lib.tff_batch_device_bytes(C.byref(self.desc)))

    def kernel_launches(self) -> int:
        return int(lib.tff_batch_kernel_launches(self._h))

    def graph_launches(self) -> int:
        """Evaluations so far that replayed a captured CUDA graph (evaluate_packed on the
        same device buffers and DFT size class as the call before captures one)."""
        return int(lib.tff_batch_graph_launches(self._h))

    def pack(self, systems: list[SystemSpec]) -> dict:
        """Device tensors of a batch (systems one after another), reusable across calls."""
        dev, dt = self.device, self.dtype
        natoms = np.array([s.natoms for s in systems], dtype=np.int64)
        grids = np.array([s.pme_grid for s in systems], dtype=np.int32)
        cat = lambda a: torch.from_numpy(np.concatenate(a)).to(dev, dt)  # noqa: E731
        return {
            "natoms": natoms, "pme_grid": grids,
            "coords": cat([s.coords.reshape(-1) for s in systems]).contiguous(),
            "boxes": cat([s.box.reshape(-1) for s in systems]).contiguous(),
            "charges": cat([s.charges for s in systems]), "sigma": cat([s.sigma for s in systems]),
            "epsilon": cat([s.epsilon for s in systems]),
            "excl": torch.from_numpy(np.concatenate([exclusion_table(s.natoms, s.excl_pairs) for s in systems])).to(dev),
            "energies": torch.empty(len(systems), dtype=torch.float64, device=dev),
            "forces": torch.empty((int(natoms.sum()), 3), dtype=dt, device=dev),
        }

    def evaluate_packed(self, p: dict) -> None:
        """Enqueue one evaluation of a packed batch on the current stream (outputs in p)."""
        nsys = len(p["natoms"])
        st = lib.tff_batch_eval(self._h, nsys, p["natoms"].ctypes.data_as(C.c_void_p),
                                p["pme_grid"].ctypes.data_as(C.c_void_p), _lib.ptr(p["coords"]), _lib.ptr(p["boxes"]),
                                _lib.ptr(p["charges"]), _lib.ptr(p["sigma"]), _lib.ptr(p["epsilon"]),
                                _lib.ptr(p["excl"]), _lib.ptr(p["energies"]), _lib.ptr(p["forces"]),
                                _lib.stream_of(p["coords"]))
        check(st, "tff_batch_eval")

    def evaluate(self, systems: list[SystemSpec]) -> tuple[torch.Tensor, list[torch.Tensor]]:
        """Energies (nsys,) float64 and per-system forces (n_i, 3) in the batch dtype."""
        p = self.pack(systems)
        self.evaluate_packed(p)
        off = np.concatenate([[0], np.cumsum(p["natoms"])])
        return p["energies"], [p["forces"][off[i]:off[i + 1]] for i in range(len(systems))]

    def status(self) -> int:
        v = C.c_int()
        check(lib.tff_batch_status(self._h, _lib.stream_of(torch.empty(0, device=self.device)), C.byref(v)),
              "tff_batch_status")
        return int(v.value)


class PreparedRequest:
    """Contiguous float64 inputs and the C request descriptor of one system."""

    def __init__(self, spec: SystemSpec):
        self.natoms = spec.natoms
        self._excl = np.ascontiguousarray(spec.excl_pairs, dtype=np.int64).reshape(-1, 2)
        self._arrays = [np.ascontiguousarray(a, dtype=np.float64) for a in
                        (spec.coords, spec.box, spec.charges, spec.sigma, spec.epsilon)]
        self.desc = _lib.RequestDesc(spec.natoms, int(spec.pme_grid), *(a.ctypes.data for a in self._arrays),
                                     self._excl.shape[0], self._excl.ctypes.data, None, None)


class ServerRequest:
    """Handle of a submitted request; energy / forces are filled in when it completes."""

    def __init__(self, server: "Server", ticket: int, energy: np.ndarray, forces: np.ndarray):
        self.server = server
        self.ticket = ticket
        self.energy = energy  # written by the server's worker thread on completion
        self.forces = forces
        self._released = False

    def done(self) -> bool:
        v = C.c_int()
        check(lib.tff_server_poll(self.server._h, self.ticket, C.byref(v)), "tff_server_poll")
        return bool(v.value)

    def wait(self, timeout: float | None = None) -> tuple[float, np.ndarray]:
        check(lib.tff_server_wait(self.server._h, self.ticket, -1.0 if timeout is None else float(timeout)),
              "tff_server_wait")
        return float(self.energy[0]), self.forces

    def times(self) -> tuple[float, float, float]:
        """(submitted, batch started, completed) on the server clock, seconds."""
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        check(lib.tff_server_request_times(self.server._h, self.ticket, C.byref(a), C.byref(b), C.byref(c)),
              "tff_server_request_times")
        return a.value, b.value, c.value

    def release(self) -> None:
        """Forget a finished request (its output arrays stay valid)."""
        if not self._released:
            check(lib.tff_server_release(self.server._h, self.ticket), "tff_server_release")
            self.server._live.pop(self.ticket, None)
            self._released = True


class Server:
    """Continuous-batching server (``tff_server``) for one cutoff / Ewald alpha."""

    def __init__(self, cutoff: float, ewald_alpha: float, dtype: torch.dtype = torch.float32, lanes: int = 3,
                 max_systems_per_batch: int = 256, hbm_budget_bytes: int = 4 << 30,
                 grid_points_per_atom: float = 16.0, coul_constant: float = 138.935456,
                 atoms_per_cell: float = 0.0, device=None):
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.desc = _lib.ServerDesc(_lib.dtype_code(dtype), int(lanes), int(max_systems_per_batch),
                                    int(hbm_budget_bytes), float(grid_points_per_atom), float(cutoff),
                                    float(ewald_alpha), float(coul_constant), float(atoms_per_cell))
        self._h = C.c_void_p()
        self._live = {}  # ticket -> request: keeps the output arrays alive until released
        with torch.cuda.device(self.device):
            check(lib.tff_server_create(C.byref(self.desc), C.byref(self._h)), "tff_server_create")

    @staticmethod
    def prepare(spec: SystemSpec) -> "PreparedRequest":
        """The request descriptor of a system, built once (submit() accepts it directly)."""
        return PreparedRequest(spec)

    def submit(self, spec) -> ServerRequest:
        """Queue one system (a SystemSpec or a PreparedRequest); inputs are copied now,
        outputs arrive in the returned request."""
        prep = spec if isinstance(spec, PreparedRequest) else PreparedRequest(spec)
        out_e = np.empty(1, dtype=np.float64)
        out_f = np.empty((prep.natoms, 3), dtype=np.float64)
        d = prep.desc
        d.energy, d.forces = out_e.ctypes.data, out_f.ctypes.data
        ticket = C.c_int64()
        check(lib.tff_server_submit(self._h, C.byref(d), C.byref(ticket)), "tff_server_submit")
        req = ServerRequest(self, int(ticket.value), out_e, out_f)
        self._live[req.ticket] = req
        return req

    def hold(self, on: bool = True) -> None:
        """While held, no new batch starts; requests keep queueing (e.g. to measure a full queue)."""
        check(lib.tff_server_hold(self._h, 1 if on else 0), "tff_server_hold")

    def drain(self, timeout: float | None = None) -> None:
        check(lib.tff_server_drain(self._h, -1.0 if timeout is None else float(timeout)), "tff_server_drain")

    def stats(self) -> dict:
        s = _lib.ServerStats()
        check(lib.tff_server_get_stats(self._h, C.byref(s)), "tff_server_get_stats")
        return {name: getattr(s, name) for name, _ in s._fields_}

    def now(self) -> float:
        return self.stats()["now"]

    def close(self) -> None:
        """Finishes the queued requests, then frees the server."""
        if self._h:
            lib.tff_server_destroy(self._h)
            self._h = C.c_void_p()
            self._live.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune_atoms_per_cell(systems: list[SystemSpec], cutoff: float, ewald_alpha: float,
                            dtype: torch.dtype = torch.float32, candidates=(5.0, 6.5, 8.0, 10.0, 12.0),
                            reps: int = 5) -> tuple[float, dict]:
    """Times one batch of `systems` at each cell occupancy; returns the fastest and all times (ms)."""
    times = {}
    natoms = sum(s.natoms for s in systems)
    grid = sum(s.pme_grid ** 3 for s in systems)
    for apc in candidates:
        ev = BatchEvaluator(cutoff, ewald_alpha, dtype, max_systems=len(systems), max_atoms=natoms,
                            max_grid_points=grid, atoms_per_cell=apc)
        p = ev.pack(systems)
        for _ in range(2):
            ev.evaluate_packed(p)
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        best = float("inf")
        for _ in range(reps):
            start.record()
            ev.evaluate_packed(p)
            end.record()
            end.synchronize()
            best = min(best, start.elapsed_time(end))
        times[apc] = best
        ev.close()
    return min(times, key=times.get), times
