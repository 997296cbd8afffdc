"""Chunk-size policy for the torch.func linearization of user residuals.

Interface of torchls ``batching.py:11-51`` (``AutoBatchSize`` with
``memory_budget_bytes`` and ``safety_factor``; ``resolve`` returns a chunk
length or None for one chunk). Chunking changes no result, only peak memory.
Built-in residuals never use it: their fused kernels take every factor in one
launch.

This package's policy sizes a chunk from what one factor occupies while its
chunk is alive on the device: its gathered inputs, the ``vmap``'d derivative
pass (one replay of the residual's intermediates, taken as proportional to
the inputs plus the output, per basis vector: r for reverse mode, D for
forward), the per-slot Jacobian blocks torch.func returns and the packed
structure-of-arrays copy the CUDA layout keeps, plus the residual. The chunk
is rounded down to a multiple of 128 factors (one linearization CTA).
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import torch

_CTA = 128


@dataclass(frozen=True)
class AutoBatchSize:
    """Chunk length from a device-memory budget (an estimate, not a limit:
    a residual function may allocate intermediates this cannot see)."""

    memory_budget_bytes: int = 256 * 1024**2
    safety_factor: float = 8.0

    def __post_init__(self):
        budget = self.memory_budget_bytes
        if isinstance(budget, bool) or not isinstance(budget, int) or budget < 1:
            raise ValueError("memory_budget_bytes must be a positive integer")
        if not (math.isfinite(self.safety_factor) and self.safety_factor >= 1):
            raise ValueError("safety_factor must be finite and at least one")

    def bytes_per_factor(self, *, input_bytes, residual_dim, tangent_dim, mode, itemsize) -> int:
        reverse = mode == "reverse" or (mode == "auto" and residual_dim <= tangent_dim)
        basis = residual_dim if reverse else tangent_dim
        replay = basis * (input_bytes + itemsize * residual_dim)
        blocks = 2 * itemsize * residual_dim * tangent_dim  # torch.func blocks + packed copy
        return input_bytes + replay + blocks + itemsize * residual_dim

    def resolve(self, *, count, input_bytes, residual_dim, tangent_dim, mode, itemsize, device):
        per = self.bytes_per_factor(input_bytes=input_bytes, residual_dim=residual_dim,
                                    tangent_dim=tangent_dim, mode=mode, itemsize=itemsize)
        budget = self.memory_budget_bytes
        if torch.device(device).type == "cuda":
            free = torch.cuda.mem_get_info(device)[0]
            budget = min(budget, max(1, free // 4))
        chunk = int(budget / (self.safety_factor * max(per, 1)))
        chunk = max(_CTA, chunk // _CTA * _CTA)
        return None if chunk >= count else chunk


BatchSize = int | AutoBatchSize | None
