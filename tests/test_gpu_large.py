"""Counts beyond 32 bits (the reference keeps counts in uint32 push constants,
src/kernel/kernel_launcher.cpp:16, :25, :1595): reduce, inclusive / exclusive scan,
copy_if and sort over 2^32 + 4097 int32 elements on the device. The all-ones input makes
every prefix known, so scans are checked exactly at sampled positions; the sort is checked
by properties that hold at any size."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = (1 << 32) + 4097


@pytest.fixture(scope="module")
def ones(dev):
    torch = dev.torch
    if torch.cuda.get_device_properties(0).total_memory < 60 << 30:
        pytest.skip("needs about 40 GB of device memory")
    x = torch.ones(N, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()  # the runtime works on its own stream
    yield x
    del x
    torch.cuda.empty_cache()


def sample_positions():
    rng = np.random.default_rng(5)
    fixed = [0, 1, 4095, 4096, (1 << 31) - 1, 1 << 31, (1 << 32) - 1, 1 << 32, N - 1]
    return np.unique(np.concatenate([fixed, rng.integers(0, N, 200)])).astype(np.int64)


def test_reduce_over_2e32(lib, px, ones):
    out = (C.c_ubyte * 4)()
    lib.parallax_reduce(px.builtin("reduce:sum:i32"), ones.data_ptr(), N, 4, out)
    px.check("reduce")
    assert np.frombuffer(bytes(out), np.uint32)[0] == N % (1 << 32)  # wraps like int32


def test_scans_over_2e32(lib, px, dev, ones):
    torch = dev.torch
    out = torch.empty(N, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    h = px.builtin("scan:i32")
    init = np.array([7], np.int32)
    lib.parallax_exclusive_scan(h, h, h, ones.data_ptr(), out.data_ptr(), N, 4, init.ctypes.data)
    px.check("exclusive scan")
    idx = sample_positions()
    got = out[torch.from_numpy(idx).cuda()].cpu().numpy().view(np.uint32)
    assert np.array_equal(got, ((idx + 7) % (1 << 32)).astype(np.uint32))
    out.copy_(ones)
    torch.cuda.synchronize()
    lib.parallax_scan(h, h, out.data_ptr(), N, 4)
    px.check("inclusive scan")
    got = out[torch.from_numpy(idx).cuda()].cpu().numpy().view(np.uint32)
    assert np.array_equal(got, ((idx + 1) % (1 << 32)).astype(np.uint32))
    del out


def test_copy_if_over_2e32(lib, px, dev, ones):
    torch = dev.torch
    out = torch.zeros(N, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    h = px.builtin("copy_if:i32:gt:0")
    k = lib.parallax_copy_if(h, h, h, h, ones.data_ptr(), out.data_ptr(), N, 4, 0)
    px.check("copy_if")
    assert k == N
    idx = sample_positions()
    assert bool((out[torch.from_numpy(idx).cuda()] == 1).all())
    h = px.builtin("copy_if:i32:lt:0")
    assert lib.parallax_copy_if(h, h, h, h, ones.data_ptr(), out.data_ptr(), N, 4, 0) == 0
    px.check("copy_if none kept")
    del out


def test_sort_over_2e32(lib, px, dev, ones):
    """Sortedness and an unchanged sum and min/max (size-independent properties) for a
    2^32 + 4097 int32 sort (about 50 GB on the device with the ones array and the sort's
    temporary)."""
    torch = dev.torch
    g = torch.Generator(device="cuda")
    g.manual_seed(9)
    x = torch.randint(-(1 << 31), (1 << 31) - 1, (N,), dtype=torch.int32, device="cuda",
                      generator=g)
    s0 = int(x.sum(dtype=torch.int64).item())
    lo, hi = int(x.min().item()), int(x.max().item())
    lib.parallax_sort(px.builtin("sort:i32"), x.data_ptr(), N, 4)
    px.check("sort")
    assert bool((x[1:] >= x[:-1]).all())
    assert int(x.sum(dtype=torch.int64).item()) == s0
    assert int(x[0].item()) == lo and int(x[-1].item()) == hi
    del x
    torch.cuda.empty_cache()
