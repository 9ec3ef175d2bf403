"""PME reciprocal space for point charges (interface of torchff/pme.py, rank 0).

Forward computes the energy (e^2/nm units; callers multiply by the Coulomb constant),
and the derivatives dE/dx and dE/dq = phi are produced in the same call, so backward
only scales them. Ranks 1 and 2 and ``return_fields`` raise NotImplementedError.
"""
from __future__ import annotations

from typing import Optional

import torch
import torch.nn as nn

from . import bsplines
from . import ops as _ops  # noqa: F401


class PME(nn.Module):
    def __init__(self, alpha: float, max_hkl: int, rank: int, use_customized_ops: bool = False,
                 return_fields: bool = False):
        super().__init__()
        if rank != 0:
            raise NotImplementedError("only rank 0 (point charges) is implemented")
        if return_fields:
            raise NotImplementedError("return_fields is not implemented")
        self.alpha = float(alpha)
        self.max_hkl = int(max_hkl)
        self.rank = int(rank)
        self.use_customized_ops = use_customized_ops
        self.return_fields = return_fields
        K = self.max_hkl
        # float64 moduli (the reference registers float32 ones, torchff/pme.py:21-28, which
        # limits its FP64 path to ~1e-7 relative); .to(float32) still casts them down.
        self.register_buffer("xmoduli", bsplines.compute_bspline_moduli_1d(K, dtype=torch.float64))
        self.register_buffer("ymoduli", bsplines.compute_bspline_moduli_1d(K, dtype=torch.float64))
        self.register_buffer("zmoduli", bsplines.compute_bspline_moduli_z(K, dtype=torch.float64))

    @torch._dynamo.disable
    def forward(self, coords: torch.Tensor, box: torch.Tensor, q: torch.Tensor, p: Optional[torch.Tensor] = None,
                t: Optional[torch.Tensor] = None):
        return torch.ops.torchff.pme_long_range(coords, box, q, p, t, self.max_hkl, self.alpha,
                                                self.xmoduli, self.ymoduli, self.zmoduli)
