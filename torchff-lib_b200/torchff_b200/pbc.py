"""Minimum-image helper (interface of torchff/pbc.py): ds - floor(ds + 0.5) in fractional space."""
from __future__ import annotations

from typing import Optional

import torch
import torch.nn as nn


def applyPBC(dr_vecs: torch.Tensor, box: Optional[torch.Tensor] = None,
             box_inv: Optional[torch.Tensor] = None) -> torch.Tensor:
    if box is not None and box_inv is None:
        box_inv, _ = torch.linalg.inv_ex(box)
    if box is None or box_inv is None:
        return dr_vecs
    ds = dr_vecs @ box_inv
    return (ds - torch.floor(ds + 0.5)) @ box


class PBC(nn.Module):
    def __init__(self, box: Optional[torch.Tensor] = None, box_inv: Optional[torch.Tensor] = None):
        super().__init__()
        if box is not None and box_inv is not None:
            self.register_buffer("box", box)
            self.register_buffer("box_inv", box_inv)
        else:
            self.box = None
            self.box_inv = None

    def forward(self, dr_vecs, box=None, box_inv=None):
        box = box if box is not None else self.box
        box_inv = box_inv if box_inv is not None else self.box_inv
        return applyPBC(dr_vecs, box, box_inv)
