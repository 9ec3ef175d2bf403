"""Shared helpers for the GPU parity tests."""
import numpy as np
import torch


def t(a, dtype=torch.float64, grad=False):
    x = torch.tensor(np.asarray(a), dtype=dtype, device="cuda")
    if grad:
        x.requires_grad_(True)
    return x


def rel_max(a, b):
    """max |a - b| / max |b| (a, b array-likes)."""
    a = a.detach().double().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a, float)
    b = b.detach().double().cpu().numpy() if isinstance(b, torch.Tensor) else np.asarray(b, float)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def rel_rms(a, b):
    a = a.detach().double().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a, float)
    b = b.detach().double().cpu().numpy() if isinstance(b, torch.Tensor) else np.asarray(b, float)
    return float(np.sqrt(np.mean((a - b) ** 2)) / np.sqrt(np.mean(b ** 2)))


def rel(a, b):
    return abs(float(a) - float(b)) / max(abs(float(b)), 1e-300)


def canon(pairs: torch.Tensor, npairs: torch.Tensor | None = None) -> np.ndarray:
    from oracle import oracle as O

    p = pairs.detach().cpu().numpy()
    if npairs is not None:
        p = p[: int(npairs.item())]
    return O.canonical_pairs(p)
