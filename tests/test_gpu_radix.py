"""The two device sort paths - merge passes (small arrays) and the one-sweep radix sort
(large arrays) - against the oracle's std::sort under the same total order, through
parallax_sort. PARALLAX_SORT forces one path, so both are checked at every size, including
the sizes where the other would be chosen: a single (ragged) radix tile, tile boundaries,
skewed digit distributions, IEEE special values and repeated calls that reuse the radix
look-back words of earlier sorts. Results are compared byte for byte."""
from __future__ import annotations

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RADIX_TILE = {4: 8192, 8: 4096}  # keys per radix tile (512 threads x 16 / 8 keys)
DTYPES = {"f32": np.float32, "f64": np.float64, "i32": np.int32, "i64": np.int64,
          "u32": np.uint32, "u64": np.uint64}


@pytest.fixture
def path():
    old = os.environ.get("PARALLAX_SORT")

    def set_path(p):
        os.environ["PARALLAX_SORT"] = p

    yield set_path
    if old is None:
        os.environ.pop("PARALLAX_SORT", None)
    else:
        os.environ["PARALLAX_SORT"] = old


def make(ox, t, n, seed):
    x = {"f32": lambda: ox.gen("f32_unit", seed, n) * 2 - 1,
         "f64": lambda: ox.gen("f64_unit", seed, n) * 2 - 1,
         "i32": lambda: ox.gen("i32_pm1000", seed, n),
         "i64": lambda: ox.gen("i64_full", seed, n),
         "u32": lambda: ox.gen("u32_full", seed, n),
         "u64": lambda: ox.gen_u64(seed, n)}[t]()
    return np.ascontiguousarray(x.astype(DTYPES[t]))


def sort_dev(lib, px, dev, t, x):
    d = dev.put(x)
    lib.parallax_sort(px.builtin(f"sort:{t}"), d.data_ptr(), x.size, x.itemsize)
    px.check("parallax_sort")
    return dev.get(d, x.dtype, x.size)


def same_bytes(a, b):
    return np.array_equal(a.view(np.uint8), b.view(np.uint8))


def sizes(es):
    tile = RADIX_TILE[es]
    return [2, 3, 17, 1000, tile - 1, tile, tile + 1, 3 * tile + 5, 100003, (1 << 20) + 3]


@pytest.mark.parametrize("algo", ["radix", "merge"])
@pytest.mark.parametrize("t", list(DTYPES))
def test_both_paths_match_oracle(lib, px, ox, dev, path, algo, t):
    path(algo)
    for i, n in enumerate(sizes(np.dtype(DTYPES[t]).itemsize)):
        x = make(ox, t, n, seed=100 + i)
        got = sort_dev(lib, px, dev, t, x)
        assert same_bytes(got, ox.sort(x)), (algo, t, n)


@pytest.mark.parametrize("t", ["f32", "f64"])
def test_ieee_special_values(lib, px, ox, dev, path, t):
    """Both signed zeros, both infinities, quiet NaNs of either sign and several payloads,
    subnormals: each path orders them by the IEEE total order, as the oracle does."""
    dt = DTYPES[t]
    specials = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, -np.nan, 1e-40 if t == "f32"
                         else 1e-310, -(1e-40 if t == "f32" else 1e-310)], dtype=dt)
    payload = (np.array([0x7fc00001, 0xffc00002, 0x7f800003], dtype=np.uint32).view(np.float32)
               if t == "f32" else
               np.array([0x7ff8000000000001, 0xfff8000000000002], dtype=np.uint64).view(np.float64))
    n = 3 * RADIX_TILE[np.dtype(dt).itemsize] + 77
    x = make(ox, t, n, seed=5)
    rng = np.random.default_rng(3)
    pool = np.concatenate([specials, payload.astype(dt)])
    pos = rng.choice(n, size=n // 5, replace=False)
    x[pos] = pool[rng.integers(0, pool.size, pos.size)]
    want = ox.sort(x)
    for algo in ("radix", "merge"):
        path(algo)
        assert same_bytes(sort_dev(lib, px, dev, t, x), want), algo
    assert np.isnan(want[0]) and np.signbit(want[0])  # a negative NaN sorts first


@pytest.mark.parametrize("t", ["u32", "i64"])
@pytest.mark.parametrize("shape", ["equal", "two_values", "sorted", "reversed", "narrow"])
def test_skewed_digit_distributions(lib, px, ox, dev, path, t, shape):
    """Every key in one digit bin (all equal), two bins, already sorted, reversed, and a
    narrow range where the high digits never change."""
    n = (1 << 19) + 9
    x = make(ox, t, n, seed=21)
    if shape == "equal":
        x[:] = x[0]
    elif shape == "two_values":
        x = np.where(x & 1, x[0], x[1]).astype(x.dtype)
    elif shape == "sorted":
        x = np.sort(x)
    elif shape == "reversed":
        x = np.sort(x)[::-1].copy()
    else:
        x = (x % 300).astype(x.dtype)
    want = ox.sort(x)
    for algo in ("radix", "merge"):
        path(algo)
        assert same_bytes(sort_dev(lib, px, dev, t, x), want), algo


def test_repeated_sorts_reuse_lookback_words(lib, px, ox, dev, path):
    """Consecutive radix sorts of shrinking and growing sizes find words of earlier passes in
    the look-back buffer; each must still read them as stale."""
    path("radix")
    for i, n in enumerate([(1 << 21) + 1, 5000, 1 << 20, 3, (1 << 22) - 7, 70000]):
        for t in ("u32", "f64"):
            x = make(ox, t, n, seed=300 + i)
            assert same_bytes(sort_dev(lib, px, dev, t, x), ox.sort(x)), (t, n)


def test_sort_kv_large_records(lib, px, ox, dev):
    """8-byte key-value records above the radix threshold: ordered by key, ties by value."""
    n = (1 << 21) + 3
    keys = (ox.gen("u32_full", 31, n) % 5000).astype(np.uint64)
    rec = (keys << np.uint64(32)) | np.arange(n, dtype=np.uint64)
    d = dev.put(rec)
    lib.parallax_sort(px.builtin("sort_kv:u32"), d.data_ptr(), n, 8)
    px.check("sort_kv")
    got = dev.get(d, np.uint64, n)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(got & np.uint64(0xFFFFFFFF), order.astype(np.uint64))
    assert np.array_equal(got >> np.uint64(32), keys[order])
