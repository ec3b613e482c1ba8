"""Synchronous scans of large coherent arena blocks: the runtime splits the tiles into chunks
and overlaps each chunk's upload and download with the tiles of its neighbours (copy
streams of the workspace). The results must be those of the oracle, as for any other scan,
for in-place and separate operands, for every element type, with one side device-resident
or a raw device pointer, and for an unaligned operand (which takes the one-launch path)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from cases import F32_TOL, F64_TOL

pytestmark = pytest.mark.gpu

DTYPES = {"f32": np.float32, "f64": np.float64, "i32": np.int32, "i64": np.int64,
          "u32": np.uint32, "u64": np.uint64}
MIN_BYTES = 64 << 20  # operands from this size up take the overlapped path


def size_for(t):
    s = np.dtype(DTYPES[t]).itemsize
    return MIN_BYTES // s + 12345  # a ragged last chunk and a ragged last tile


def gen(ox, t, n, seed):
    return {"f32": lambda: ox.gen("f32_unit", seed, n), "f64": lambda: ox.gen("f64_unit", seed, n),
            "i32": lambda: ox.gen("i32_pm1000", seed, n), "i64": lambda: ox.gen("i64_full", seed, n),
            "u32": lambda: ox.gen("u32_full", seed, n), "u64": lambda: ox.gen_u64(seed, n)}[t]()


def same(t, got, want):
    if t == "f32":
        return np.max(np.abs(got.astype(np.float64) - want) / np.maximum(np.abs(want), 1e-30)) <= F32_TOL
    if t == "f64":
        return np.max(np.abs(got - want) / np.maximum(np.abs(want), 1e-300)) <= F64_TOL
    return np.array_equal(got, want)


class Blocks:
    def __init__(self, lib):
        self.lib, self.ptrs = lib, []

    def array(self, a, extra=0):
        p = self.lib.parallax_arena_alloc(a.nbytes + extra, 256)
        assert p, "arena_alloc failed"
        self.ptrs.append(p)
        v = np.ctypeslib.as_array((C.c_ubyte * (a.nbytes + extra)).from_address(p))
        v = v[extra: extra + a.nbytes].view(a.dtype)
        v[:] = a
        return v

    def free(self):
        for p in self.ptrs:
            self.lib.parallax_arena_free(p)


@pytest.fixture
def blocks(lib):
    b = Blocks(lib)
    yield b
    b.free()


@pytest.mark.parametrize("t", list(DTYPES))
def test_inclusive_in_place(lib, px, ox, blocks, t):
    n = size_for(t)
    x = gen(ox, t, n, seed=61)
    data = blocks.array(x)
    h = px.builtin(f"scan:{t}")
    lib.parallax_scan(h, h, data.ctypes.data, n, x.itemsize)
    px.check("scan")
    assert same(t, data.copy(), ox.scan(x))


@pytest.mark.parametrize("t", ["f32", "i32", "i64", "u64"])
def test_exclusive_separate_blocks(lib, px, ox, blocks, t):
    n = size_for(t)
    x = gen(ox, t, n, seed=62)
    src = blocks.array(x)
    dst = blocks.array(np.zeros_like(x))
    h = px.builtin(f"scan:{t}")
    init = np.array([5], dtype=x.dtype)
    lib.parallax_exclusive_scan(h, h, h, src.ctypes.data, dst.ctypes.data, n, x.itemsize,
                                init.ctypes.data)
    px.check("exclusive scan")
    assert same(t, dst.copy(), ox.scan(x, exclusive=True, init=5))
    assert np.array_equal(src, x)  # the input is left as it was


def test_exclusive_device_resident_input(lib, px, ox, blocks):
    t, n = "i32", size_for("i32")
    x = gen(ox, t, n, seed=63)
    src = blocks.array(x)
    lib.parallax_arena_set_residency(src.ctypes.data, px.DEVICE_RESIDENT)
    lib.parallax_arena_sync_to_device(src.ctypes.data, x.nbytes)
    src[:] = 0  # the host mirror no longer matters
    dst = blocks.array(np.zeros_like(x))
    h = px.builtin("scan:i32")
    lib.parallax_exclusive_scan(h, h, h, src.ctypes.data, dst.ctypes.data, n, 4, None)
    px.check("exclusive scan")
    assert np.array_equal(dst, ox.scan(x, exclusive=True, init=0))


def test_exclusive_into_device_pointer(lib, px, ox, dev, blocks):
    t, n = "i64", size_for("i64")
    x = gen(ox, t, n, seed=64)
    src = blocks.array(x)
    out = dev.empty(x.nbytes)
    dev.torch.cuda.synchronize()
    h = px.builtin("scan:i64")
    lib.parallax_exclusive_scan(h, h, h, src.ctypes.data, out.data_ptr(), n, 8, None)
    px.check("exclusive scan")
    assert np.array_equal(dev.get(out, np.int64, n), ox.scan(x, exclusive=True, init=0))


def test_unaligned_operand_takes_one_launch(lib, px, ox, blocks):
    t, n = "u32", size_for("u32")
    x = gen(ox, t, n, seed=65)
    data = blocks.array(x, extra=4)  # 4 bytes past a 256-byte boundary
    h = px.builtin("scan:u32")
    lib.parallax_scan(h, h, data.ctypes.data, n, 4)
    px.check("scan")
    assert np.array_equal(data, ox.scan(x))


def test_repeated_calls_and_growth(lib, px, ox, blocks):
    """Back-to-back overlapped scans of growing sizes reuse the copy streams and events."""
    h = px.builtin("scan:i32")
    for i, n in enumerate([size_for("i32"), 3 * size_for("i32") + 1, size_for("i32") + 7]):
        x = gen(ox, "i32", n, seed=70 + i)
        data = blocks.array(x)
        lib.parallax_scan(h, h, data.ctypes.data, n, 4)
        px.check("scan")
        assert np.array_equal(data, ox.scan(x)), n
