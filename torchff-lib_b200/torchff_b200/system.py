"""Fused fixed-charge nonbonded evaluation of one periodic system.

``FixedChargeSystem`` owns a libtffb200 system object: per-atom charges, Lennard-Jones
sigma/epsilon (Lorentz-Berthelot combining), the exclusion list, a PME plan and all
scratch, resident on the device. One ``evaluate`` call rebuilds the cluster-pair
neighbour structure from the coordinates and returns the energy

    E = sum_{pairs, r<=rc} [4 eps_ij((s_ij/r)^12 - (s_ij/r)^6) + k q_i q_j erfc(a r)/r]
        - sum_{excluded pairs, r<=rc} k q_i q_j erf(a r)/r
        + k E_pme(a, K)

and forces, i.e. the nonbonded part of ``Tip3pTorchFF`` (examples/tip3p/model.py:100-133:
NeighborList + Vdw + MultipolarInteraction(rank 0, pairs_excl) + 138.935456 * PME), with
excluded pairs removed from the neighbour list and given the Ewald exclusion correction.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch
import torch.nn as nn

from . import _lib as L

COULOMB_PREFACTOR = 138.935456


class FixedChargeSystem:
    def __init__(self, charges, sigma, epsilon, exclusions, cutoff: float, ewald_alpha: float, pme_grid: int,
                 coul_constant: float = COULOMB_PREFACTOR, dtype: torch.dtype = torch.float32,
                 device: torch.device | str = "cuda", max_cluster_neighbors: int = 0, check_status: bool = False):
        """check_status: after every evaluate() / evaluate_grads() (and so every module
        forward), wait for the device and raise if a cluster's neighbour list overflowed its
        capacity (pairs dropped). Off by default: the check synchronises. evaluate_host
        always checks (it synchronises anyway); evaluate_into never does (graph capture)."""
        self.check_status = bool(check_status)
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise RuntimeError("FixedChargeSystem needs a CUDA device")
        self.dtype = dtype
        q = np.ascontiguousarray(np.asarray(charges, dtype=np.float64).reshape(-1))
        s = np.ascontiguousarray(np.asarray(sigma, dtype=np.float64).reshape(-1))
        e = np.ascontiguousarray(np.asarray(epsilon, dtype=np.float64).reshape(-1))
        ex = np.ascontiguousarray(np.asarray(exclusions if exclusions is not None else np.zeros((0, 2)),
                                             dtype=np.int64).reshape(-1, 2))
        self.natoms = int(q.shape[0])
        if s.shape[0] != self.natoms or e.shape[0] != self.natoms:
            raise ValueError("charges, sigma and epsilon must all have natoms entries")
        self.cutoff, self.ewald_alpha, self.pme_grid = float(cutoff), float(ewald_alpha), int(pme_grid)
        self.coul_constant = float(coul_constant)
        desc = L.SystemDesc(L.dtype_code(dtype), self.natoms, self.cutoff, self.ewald_alpha, self.pme_grid,
                            self.coul_constant, int(max_cluster_neighbors))
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            L.check(L.lib.tff_system_create(ctypes.byref(desc), q.ctypes.data_as(ctypes.c_void_p),
                                            s.ctypes.data_as(ctypes.c_void_p), e.ctypes.data_as(ctypes.c_void_p),
                                            ex.shape[0], ex.ctypes.data_as(ctypes.c_void_p), ctypes.byref(h)),
                    "tff_system_create")
        self._h = h
        # the parameters the system holds (system dtype), for callers that pass none
        self.defaults = {k: torch.tensor(v, dtype=dtype, device=self.device) for k, v in
                         (("charges", q), ("sigma", s), ("epsilon", e))}

    @classmethod
    def from_water_box(cls, wb, dtype=torch.float32, device="cuda", flexible: bool = False, **kw):
        """System for a ``torchff_b200.water.WaterBox`` (TIP3P parameters and exclusions);
        ``flexible`` adds the harmonic O-H bonds and H-O-H angles of flexible TIP3P."""
        sys_ = cls(wb.charges, wb.sigma, wb.epsilon, wb.coulomb_exclusions, wb.cutoff, wb.alpha, wb.grid,
                   dtype=dtype, device=device, **kw)
        if flexible:
            from .water import water_bonded_terms
            bt = water_bonded_terms(wb.n_waters)
            sys_.set_bonded(bt.bonds, bt.b0, bt.kb, bt.angles, bt.th0, bt.kth)
        return sys_

    def set_bonded(self, bonds=None, b0=None, kb=None, angles=None, theta0=None, ktheta=None) -> None:
        """Harmonic bonds (M,2) with b0, kb and angles (M,3) with theta0, ktheta (central atom
        in the middle) evaluated with the nonbonded terms (examples/tip3p/model.py:105-106).
        All None removes them. Synchronises the device."""
        def arr(a, dt, shape=None):
            a = np.ascontiguousarray(np.asarray(a.detach().cpu() if isinstance(a, torch.Tensor) else a, dtype=dt))
            return a if shape is None else a.reshape(shape)
        nb = na = 0
        bd = b0a = kba = an = t0a = kta = None
        if bonds is not None:
            bd = arr(bonds, np.int64, (-1, 2)); b0a = arr(b0, np.float64, -1); kba = arr(kb, np.float64, -1)
            nb = bd.shape[0]
            if b0a.shape[0] != nb or kba.shape[0] != nb:
                raise ValueError("b0 and kb need one value per bond")
        if angles is not None:
            an = arr(angles, np.int64, (-1, 3)); t0a = arr(theta0, np.float64, -1); kta = arr(ktheta, np.float64, -1)
            na = an.shape[0]
            if t0a.shape[0] != na or kta.shape[0] != na:
                raise ValueError("theta0 and ktheta need one value per angle")
        p = lambda a: None if a is None else a.ctypes.data_as(ctypes.c_void_p)
        with torch.cuda.device(self.device):
            L.check(L.lib.tff_system_set_bonded(self._h, nb, p(bd), p(b0a), p(kba), na, p(an), p(t0a), p(kta)),
                    "tff_system_set_bonded")
        self.nbonded_terms = nb + na

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                L.lib.tff_system_destroy(h)
            except Exception:
                pass
            self._h = None

    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def set_parameters(self, charges=None, sigma=None, epsilon=None) -> None:
        ts = [None if t is None else t.detach().to(self.device, self.dtype).contiguous() for t in
              (charges, sigma, epsilon)]
        L.check(L.lib.tff_system_set_parameters(self._h, *(L.ptr(t) for t in ts), self._stream()),
                "tff_system_set_parameters")

    def evaluate_into(self, coords: torch.Tensor, box: torch.Tensor, energy: torch.Tensor, forces: torch.Tensor,
                      grad_charges: torch.Tensor | None = None, energy_terms: torch.Tensor | None = None) -> None:
        """Enqueues one evaluation writing into preallocated outputs (CUDA-graph friendly).

        coords (N,3) and box (3,3) in the system dtype; energy: float64 (1,); forces (N,3)
        system dtype (= -dE/dx); grad_charges (N,) dE/dq; energy_terms float64 (4,):
        real-space pairs, exclusion correction, reciprocal, self; (6,) with bonded terms
        (then bonds, angles).
        """
        L.check(L.lib.tff_system_eval(self._h, L.ptr(coords), L.ptr(box), L.ptr(energy), L.ptr(forces),
                                      L.ptr(grad_charges), L.ptr(energy_terms), self._stream()), "tff_system_eval")

    def evaluate(self, coords: torch.Tensor, box: torch.Tensor, grad_charges: bool = False, terms: bool = False):
        x = coords.detach().to(self.device, self.dtype).contiguous()
        b = box.detach().to(self.device, self.dtype).contiguous()
        if x.shape != (self.natoms, 3):
            raise ValueError(f"coords must be ({self.natoms}, 3)")
        energy = torch.empty(1, dtype=torch.float64, device=self.device)
        forces = torch.empty_like(x)
        gq = torch.empty(self.natoms, dtype=self.dtype, device=self.device) if grad_charges else None
        et = torch.empty(6 if getattr(self, "nbonded_terms", 0) else 4, dtype=torch.float64,
                         device=self.device) if terms else None
        self.evaluate_into(x, b, energy, forces, gq, et)
        self._check_overflow()
        out = {"energy": energy[0], "forces": forces}
        if gq is not None:
            out["grad_charges"] = gq
        if et is not None:
            out["terms"] = et
        return out

    def evaluate_host(self, coords: np.ndarray | torch.Tensor, box: np.ndarray | torch.Tensor,
                      forces_out: np.ndarray | torch.Tensor) -> float:
        """Host buffers in and out (float64): H2D copy, evaluation, D2H copy, synchronise."""
        e = ctypes.c_double(0.0)
        cp = coords.data_ptr() if isinstance(coords, torch.Tensor) else coords.ctypes.data
        bp = box.data_ptr() if isinstance(box, torch.Tensor) else box.ctypes.data
        fp = forces_out.data_ptr() if isinstance(forces_out, torch.Tensor) else forces_out.ctypes.data
        L.check(L.lib.tff_system_eval_host(self._h, ctypes.c_void_p(cp), ctypes.c_void_p(bp), ctypes.byref(e),
                                           ctypes.c_void_p(fp), self._stream()), "tff_system_eval_host")
        return e.value

    def evaluate_grads(self, coords: torch.Tensor, box: torch.Tensor) -> dict:
        """Energy, forces and first derivatives with respect to the per-atom parameters
        (dE/dq, dE/dsigma, dE/depsilon; dE/deps_i = 0 where eps_i = 0)."""
        x = coords.detach().to(self.device, self.dtype).contiguous()
        b = box.detach().to(self.device, self.dtype).contiguous()
        n = self.natoms
        out = {"energy": torch.empty(1, dtype=torch.float64, device=self.device),
               "forces": torch.empty_like(x)}
        for k in ("grad_charges", "grad_sigma", "grad_epsilon"):
            out[k] = torch.empty(n, dtype=self.dtype, device=self.device)
        L.check(L.lib.tff_system_eval_grads(self._h, L.ptr(x), L.ptr(b), L.ptr(out["energy"]), L.ptr(out["forces"]),
                                            L.ptr(out["grad_charges"]), L.ptr(out["grad_sigma"]),
                                            L.ptr(out["grad_epsilon"]), self._stream()), "tff_system_eval_grads")
        self._check_overflow()
        out["energy"] = out["energy"][0]
        return out

    def _check_overflow(self) -> None:
        if self.check_status and self.status() & 1:
            raise RuntimeError("FixedChargeSystem: a cluster's neighbour list overflowed its capacity "
                               "(max_cluster_neighbors); pairs were dropped")

    def hvp(self, coords: torch.Tensor, box: torch.Tensor, direction: torch.Tensor) -> dict:
        """Derivatives of s = sum_i u_i . dE/dx_i (u = `direction`, (N,3)) with respect to the
        coordinates, charges, sigma and epsilon: one Hessian-vector product."""
        x = coords.detach().to(self.device, self.dtype).contiguous()
        b = box.detach().to(self.device, self.dtype).contiguous()
        u = direction.detach().to(self.device, self.dtype).contiguous()
        n = self.natoms
        out = {"coords": torch.empty_like(x)}
        for k in ("charges", "sigma", "epsilon"):
            out[k] = torch.empty(n, dtype=self.dtype, device=self.device)
        L.check(L.lib.tff_system_hvp(self._h, L.ptr(x), L.ptr(b), L.ptr(u), L.ptr(out["coords"]),
                                     L.ptr(out["charges"]), L.ptr(out["sigma"]), L.ptr(out["epsilon"]),
                                     self._stream()), "tff_system_hvp")
        return out

    def status(self) -> int:
        v = ctypes.c_int(0)
        L.check(L.lib.tff_system_status(self._h, self._stream(), ctypes.byref(v)), "tff_system_status")
        return v.value

    def kernel_launches(self) -> int:
        """Kernels of libtffb200 one evaluation launches (cuFFT's not counted)."""
        return int(L.lib.tff_system_kernel_launches(self._h))

    def evaluate_timed_into(self, coords, box, energy, forces, timer: "StageTimer") -> None:
        """Like evaluate_into, recording the stage events of ``timer`` (graph-capturable)."""
        L.check(L.lib.tff_system_eval_timed(self._h, L.ptr(coords), L.ptr(box), L.ptr(energy), L.ptr(forces),
                                            timer.handle, self._stream()), "tff_system_eval_timed")


class StageTimer:
    """CUDA events at the stage boundaries of a fused evaluation.

    Event k: 0 start, 1 cluster build done, 2 real-space tile kernel done (caller stream);
    3 PME grid phase done (spread, FFTs, influence function), 4 PME gather done (PME
    stream, forked at event 0); 5 finalize done (after both branches joined).
    """

    STAGES = ("cluster_build", "tile_kernel", "pme_grid", "pme_gather", "finalize", "total")

    def __init__(self):
        h = ctypes.c_void_p()
        L.check(L.lib.tff_timer_create(ctypes.byref(h)), "tff_timer_create")
        self.handle = h

    def elapsed_ms(self, a: int, b: int) -> float:
        v = ctypes.c_float(0.0)
        L.check(L.lib.tff_timer_elapsed_ms(self.handle, a, b, ctypes.byref(v)), "tff_timer_elapsed_ms")
        return float(v.value)

    def stages_ms(self) -> dict:
        out = {"cluster_build": self.elapsed_ms(0, 1), "tile_kernel": self.elapsed_ms(1, 2),
               "pme_grid": self.elapsed_ms(0, 3), "pme_gather": self.elapsed_ms(3, 4)}
        out["finalize"] = min(self.elapsed_ms(2, 5), self.elapsed_ms(4, 5))
        out["total"] = self.elapsed_ms(0, 5)
        return out

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                L.lib.tff_timer_destroy(h)
            except Exception:
                pass
            self.handle = None


class _SystemGradFn(torch.autograd.Function):
    """(coords, charges, sigma, epsilon) -> (dE/dx, dE/dq, dE/dsigma, dE/deps), values computed
    by the forward evaluation; its backward is the Hessian-vector product along the
    cotangent of dE/dx (what a force-matching loss needs)."""

    @staticmethod
    def forward(ctx, coords, box, q, sig, eps, gx, gq, gs, ge, system):
        ctx.save_for_backward(coords, box, q, sig, eps)
        ctx.system = system
        return gx.clone(), gq.clone(), gs.clone(), ge.clone()

    @staticmethod
    def backward(ctx, vx, vq, vs, ve):
        for v in (vq, vs, ve):
            if v is not None and bool(torch.any(v != 0)):
                raise NotImplementedError("second derivatives along charge/sigma/epsilon directions are not "
                                          "implemented; differentiate dE/dx only (force matching)")
        coords, box, q, sig, eps = ctx.saved_tensors
        system = ctx.system
        if vx is None:
            return (None,) * 10
        system.set_parameters(q, sig, eps)
        h = system.hvp(coords, box, vx)
        cast = lambda t, ref: t.to(ref.dtype)  # noqa: E731
        return (cast(h["coords"], coords), None, cast(h["charges"], q), cast(h["sigma"], sig),
                cast(h["epsilon"], eps), None, None, None, None, None)


class _SystemEnergyFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coords, box, q, sig, eps, system: FixedChargeSystem):
        system.set_parameters(q, sig, eps)
        if ctx.needs_input_grad[3] or ctx.needs_input_grad[4]:
            out = system.evaluate_grads(coords, box)
            gs, ge = out["grad_sigma"], out["grad_epsilon"]
        else:
            out = system.evaluate(coords, box, grad_charges=True)
            gs = ge = torch.zeros(system.natoms, dtype=system.dtype, device=system.device)
        gx = (-out["forces"]).to(coords.dtype)
        ctx.save_for_backward(coords, box, q, sig, eps, gx, out["grad_charges"].to(q.dtype), gs.to(sig.dtype),
                              ge.to(eps.dtype))
        ctx.system = system
        return out["energy"].to(coords.dtype)

    @staticmethod
    def backward(ctx, g):
        coords, box, q, sig, eps, gx, gq, gs, ge = ctx.saved_tensors
        dx, dq, ds, de = _SystemGradFn.apply(coords, box, q, sig, eps, gx, gq, gs, ge, ctx.system)
        return g * dx, None, g * dq, g * ds, g * de, None


class FixedChargeNonbonded(nn.Module):
    """nn.Module view of a FixedChargeSystem: ``forward(coords, box, charges, sigma, epsilon) -> E``.

    Forces and parameter gradients come from autograd, and the backward is itself
    differentiable along dE/dx: a loss on the forces (force matching) back-propagates to
    coordinates, charges, sigma and epsilon through one Hessian-vector product. Parameters
    left as None are the system's own.
    """

    def __init__(self, system: FixedChargeSystem):
        super().__init__()
        self.system = system

    def forward(self, coords: torch.Tensor, box: torch.Tensor, charges: torch.Tensor | None = None,
                sigma: torch.Tensor | None = None, epsilon: torch.Tensor | None = None):
        d = self.system.defaults
        q = d["charges"] if charges is None else charges
        s = d["sigma"] if sigma is None else sigma
        e = d["epsilon"] if epsilon is None else epsilon
        return _SystemEnergyFn.apply(coords, box, q, s, e, self.system)
