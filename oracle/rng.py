"""Seeded standard-normal draws, the same stream as the reference's ``seeded_randn``.

``src/cdft/precision.py:246-263`` draws from a ``torch.Generator`` on the CPU and then moves the
result; drawing with the same generator here is the only way a seeded oracle solve starts from the
same block as the reference. torch is used for nothing else in the oracle.
"""

from __future__ import annotations

import numpy as np
import torch


def make_generator(seed: int) -> torch.Generator:
    return torch.Generator(device="cpu").manual_seed(int(seed))


def seeded_randn(shape, generator) -> np.ndarray:
    size = (shape,) if isinstance(shape, int) else tuple(shape)
    return torch.randn(size, dtype=torch.float64, generator=generator).numpy().copy()
