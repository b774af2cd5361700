"""Packed-state helpers shared by the host and the library (the reference's ``device.py``).

The reference builds a constant blob for its NVRTC module here (``device.py:22-141``); in this
package libccs derives its device constants itself, so only the state packing remains.
"""

from __future__ import annotations

import numpy as np

from cuda_cube_solver import coords
from cuda_cube_solver.cubie import CubieState


def pack_states(corners: np.ndarray, edges: np.ndarray) -> np.ndarray:
    """(n, 8) and (n, 12) packed bytes -> (n, 5) uint32 words (corner bytes, then edge bytes)."""

    words = np.concatenate([np.asarray(corners), np.asarray(edges)], axis=-1).astype(np.uint8)
    return np.ascontiguousarray(words).view(np.uint32).reshape(-1, 5)


def state_words(states) -> np.ndarray:
    """Packed words of a list of ``CubieState`` (n, 5)."""

    if isinstance(states, CubieState):
        states = [states]
    packed = [coords.pack(s) for s in states]
    if not packed:
        return np.zeros((0, 5), np.uint32)
    return pack_states(np.stack([p[0] for p in packed]), np.stack([p[1] for p in packed]))


def unpack_words(words: np.ndarray) -> list[CubieState]:
    b = np.ascontiguousarray(words, dtype=np.uint32).reshape(-1, 5).view(np.uint8).reshape(-1, 20)
    return [coords.unpack(row[:8], row[8:]) for row in b]
