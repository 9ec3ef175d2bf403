"""Float64 torch restatement of the fused fixed-charge energy (TEST INFRASTRUCTURE ONLY).

The oracle for derivatives beyond first order: torch autograd of this function gives the
forces, the per-atom parameter gradients and the double backward of a force-matching loss,
which the CUDA second-derivative pass (``tff_system_hvp``) is checked against. Only the
test-suite may import it. It follows the same reference code as ``oracle.py``:

* LJ 12-6 with Lorentz-Berthelot combining of per-atom sigma/epsilon
  (``csrc/nonbonded/nonbonded_atom_pairs_cuda.cu:86-90``, ``torchff/vdw.py:86-111``);
  sqrt(eps_i eps_j) is taken as 0 with zero gradient where the product is 0 (the
  convention of the CUDA path: dE/deps_i = 0 where eps_i = 0);
* real-space Ewald k q_i q_j erfc(a r)/r on the pair list and -k q_i q_j erf(a r)/r on
  excluded pairs within the cutoff (``torchff/multipoles.py:244-341``);
* rank-0 smooth PME with order-6 B-splines from the Essmann recursion, torch FFT,
  E = 1/2 sum_k C(k) |S(k)|^2 / theta(k)^2 - (a/sqrt(pi)) sum q^2
  (``torchff/pme_ref.py:11-469``), scaled by k.

The pair list is fixed by the caller (pairs within the cutoff at the base coordinates),
so derivatives are those of a smooth function of the inputs.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from .oracle import bspline_moduli, signed_frequency


def _bspline6(u: torch.Tensor) -> torch.Tensor:
    def m(n, x):
        if n == 2:
            return torch.where((x >= 0) & (x <= 2), 1.0 - torch.abs(x - 1.0), torch.zeros_like(x))
        return (x * m(n - 1, x) + (n - x) * m(n - 1, x - 1.0)) / (n - 1)

    return torch.where((u >= 0) & (u < 6), m(6, u), torch.zeros_like(u))


def _min_image(d: torch.Tensor, box: torch.Tensor, inv: torch.Tensor) -> torch.Tensor:
    f = d @ inv
    f = f - torch.floor(f + 0.5).detach()
    return f @ box


def real_space(x, box, q, sig, eps, pairs, excl, cutoff, alpha, kc):
    inv = torch.linalg.inv(box)
    i, j = pairs[:, 0], pairs[:, 1]
    d = _min_image(x[i] - x[j], box, inv)
    r = torch.sqrt(torch.sum(d * d, 1))
    sij = 0.5 * (sig[i] + sig[j])
    prod = eps[i] * eps[j]
    pos = prod > 0
    eij = torch.where(pos, torch.sqrt(torch.where(pos, prod, torch.ones_like(prod))), torch.zeros_like(prod))
    s6 = (sij / r) ** 6
    e = torch.sum(4.0 * eij * (s6 * s6 - s6) + kc * q[i] * q[j] * torch.erfc(alpha * r) / r)
    if excl is not None and len(excl):
        a, b = excl[:, 0], excl[:, 1]
        de = _min_image(x[a] - x[b], box, inv)
        re = torch.sqrt(torch.sum(de * de, 1))
        inside = (re <= cutoff).detach()
        e = e - torch.sum(torch.where(inside, kc * q[a] * q[b] * torch.erf(alpha * re) / re, torch.zeros_like(re)))
    return e


def pme(x, box, q, alpha, K, kc):
    n = x.shape[0]
    inv = torch.linalg.inv(box)
    recip = K * inv.T                      # row d: K * inv(box)[:, d]
    frac = x @ recip.T
    m0 = torch.ceil(frac).detach()
    shifts = torch.arange(-3, 3, dtype=x.dtype)
    u = (m0 - frac + 3.0)[:, :, None] + shifts[None, None, :]
    w = _bspline6(u)                       # (N, 3, 6)
    idx = (m0.long()[:, :, None] + shifts.long()[None, None, :]) % K
    w3 = w[:, 0, :, None, None] * w[:, 1, None, :, None] * w[:, 2, None, None, :]
    flat = idx[:, 0, :, None, None] * K * K + idx[:, 1, None, :, None] * K + idx[:, 2, None, None, :]
    grid = torch.zeros(K * K * K, dtype=x.dtype).index_add(0, flat.reshape(-1), (q[:, None, None, None] * w3).reshape(-1))
    S = torch.fft.fftn(grid.reshape(K, K, K))
    bx = box.detach().numpy()
    f = signed_frequency(K).astype(np.float64)
    mx, my, mz = np.meshgrid(f, f, f, indexing="ij")
    kvec = 2.0 * np.pi * (np.stack([mx, my, mz], -1) @ np.linalg.inv(bx).T)
    ksq = np.sum(kvec * kvec, -1)
    th = bspline_moduli(K)
    theta = th[:, None, None] * th[None, :, None] * th[None, None, :]
    with np.errstate(divide="ignore", invalid="ignore"):
        C = 4.0 * np.pi / abs(np.linalg.det(bx)) / ksq * np.exp(-ksq / (4.0 * alpha * alpha)) / (theta * theta)
    C[0, 0, 0] = 0.0
    e_rec = 0.5 * torch.sum(torch.from_numpy(C) * (S.real ** 2 + S.imag ** 2))
    e_self = -alpha / math.sqrt(math.pi) * torch.sum(q * q)
    return kc * (e_rec + e_self)


def fixed_charge_energy(x, box, q, sig, eps, pairs, excl, cutoff, alpha, K, kc=138.935456):
    """Total energy (float64 scalar tensor); x, q, sig, eps may require grad."""
    return real_space(x, box, q, sig, eps, pairs, excl, cutoff, alpha, kc) + pme(x, box, q, alpha, K, kc)
