"""Chunk size policy for torch.func linearization of user residuals.

Interface of torchls ``batching.py:11-51``. Only user-defined residuals are
chunked; the built-in fused kernels process every factor in one launch.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import torch


@dataclass(frozen=True)
class AutoBatchSize:
    """Estimate a vmap chunk size from a memory budget (a heuristic, not a limit)."""

    memory_budget_bytes: int = 256 * 1024**2
    safety_factor: float = 8.0

    def __post_init__(self):
        if (isinstance(self.memory_budget_bytes, bool) or not isinstance(self.memory_budget_bytes, int)
                or self.memory_budget_bytes < 1):
            raise ValueError("memory_budget_bytes must be a positive integer")
        if not math.isfinite(self.safety_factor) or self.safety_factor < 1:
            raise ValueError("safety_factor must be finite and at least one")

    def resolve(self, *, count, input_bytes, residual_dim, tangent_dim, mode, itemsize, device):
        width = residual_dim if mode == "reverse" or (mode == "auto" and residual_dim <= tangent_dim) else tangent_dim
        row = input_bytes + itemsize * (residual_dim * (tangent_dim + 1) + tangent_dim + width * width)
        budget = self.memory_budget_bytes
        if device.type == "cuda":
            free, _ = torch.cuda.mem_get_info(device)
            budget = min(budget, max(1, free // 4))
        chunk = max(1, int(budget / max(1, row) / self.safety_factor))
        return None if chunk >= count else chunk


BatchSize = int | AutoBatchSize | None
