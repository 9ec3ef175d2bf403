"""Order-6 B-spline moduli for PME (interface of torchff/bsplines.py).

theta(k) = sum_{m=-3}^{2} M6(m + 3) cos(2 pi m k / K), with M6 at the integers from the
cardinal B-spline recursion of Essmann et al. (1995), eq. 4.1.
"""
from __future__ import annotations

import math

import torch


def _m6_at_integers() -> list[float]:
    m = [0.0, 1.0, 0.0, 0.0, 0.0, 0.0]          # M2(0), M2(1)
    for n in range(3, 7):
        m = [((k * (m[k] if k < n - 1 else 0.0)) + (n - k) * (m[k - 1] if k > 0 else 0.0)) / (n - 1)
             if k < n else 0.0 for k in range(6)]
    return m


def get_bspline_modulus(k: torch.Tensor, K: int, order: int = 6) -> torch.Tensor:
    if order != 6:
        raise ValueError("Only order=6 is implemented.")
    b = _m6_at_integers()
    kf = k.to(torch.float64)
    out = torch.zeros(kf.shape, dtype=torch.float64, device=k.device)
    for m in range(-3, 3):
        out += b[m + 3] * torch.cos(2.0 * math.pi * m * kf / K)
    return out


def compute_bspline_moduli_1d(K: int, dtype: torch.dtype = torch.float32, device=None) -> torch.Tensor:
    k = torch.arange(K, dtype=torch.int64, device=device)
    return get_bspline_modulus(k, K).to(dtype=dtype, device=device)


def compute_bspline_moduli_z(K3: int, dtype: torch.dtype = torch.float32, device=None) -> torch.Tensor:
    k = torch.arange(K3 // 2 + 1, dtype=torch.int64, device=device)
    return get_bspline_modulus(k, K3).to(dtype=dtype, device=device)
