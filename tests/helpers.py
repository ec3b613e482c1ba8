"""Helpers shared by the GPU tests."""
from __future__ import annotations

import ctypes as C

import numpy as np


class Arena:
    """numpy views of parallax_arena_alloc blocks (host addresses in the pinned mirror)."""

    def __init__(self, lib):
        self.lib = lib
        self.blocks = []

    def array(self, a: np.ndarray) -> np.ndarray:
        p = self.lib.parallax_arena_alloc(max(a.nbytes, 1), 256)
        assert p, "arena_alloc failed"
        self.blocks.append(p)
        v = np.ctypeslib.as_array((C.c_ubyte * max(a.nbytes, 1)).from_address(p))
        v = v[: a.nbytes].view(a.dtype)
        v[:] = a
        return v

    def empty(self, n: int, dtype) -> np.ndarray:
        return self.array(np.zeros(n, dtype))

    def free(self):
        for p in self.blocks:
            self.lib.parallax_arena_free(p)
        self.blocks = []
