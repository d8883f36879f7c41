"""Seeded random starts, drawn once and kept on the device.

The reference draws every random start from a CPU ``torch.Generator`` and moves it to the device
(``src/cdft/precision.py:246-263``), and its SCF re-seeds a fresh generator with the same seed in
every diagonalisation (``src/cdft/scf/step.py:338``). The draws of a diagonalisation therefore depend
only on the seed and on the sequence of shapes drawn so far, and repeat exactly from one SCF
iteration to the next. :class:`SeededStream` is a drop-in for such a freshly seeded generator: the
first time a (seed, draw sequence) occurs it draws on the CPU exactly as the reference does and
keeps the result on the device; afterwards it serves the same bits without touching the host.
"""

from __future__ import annotations

from collections import OrderedDict

import torch

#: Device bytes the cache may hold before the least recently used draws are dropped.
CACHE_BYTES = 4 << 30

_CACHE: "OrderedDict[tuple, torch.Tensor]" = OrderedDict()
_CACHE_SIZE = [0]


class SeededStream:
    """A freshly seeded CPU generator whose draws are cached on ``device`` (see module doc)."""

    def __init__(self, seed: int, device: torch.device | str) -> None:
        self.seed = int(seed)
        self.device = torch.device(device)
        self._history: tuple = ()
        self._generator: torch.Generator | None = None

    def _replay(self) -> torch.Generator:
        # A real generator advanced through the draws made so far (only on a cache miss).
        g = torch.Generator(device="cpu").manual_seed(self.seed)
        for shape in self._history:
            torch.randn(shape, dtype=torch.float64, generator=g)
        return g

    def randn(self, shape) -> torch.Tensor:
        size = (shape,) if isinstance(shape, int) else tuple(shape)
        key = (self.seed, str(self.device), self._history, size)
        hit = _CACHE.get(key)
        if hit is None:
            g = self._generator if self._generator is not None else self._replay()
            draw = torch.randn(size, dtype=torch.float64, generator=g)
            self._generator = g
            hit = draw.to(self.device)
            _CACHE[key] = hit
            _CACHE_SIZE[0] += hit.numel() * 8
            while _CACHE_SIZE[0] > CACHE_BYTES and len(_CACHE) > 1:
                _, old = _CACHE.popitem(last=False)
                _CACHE_SIZE[0] -= old.numel() * 8
        else:
            _CACHE.move_to_end(key)
            self._generator = None  # a later miss replays from the seed
        self._history = self._history + (size,)
        return hit


def clear_cache() -> None:
    _CACHE.clear()
    _CACHE_SIZE[0] = 0
