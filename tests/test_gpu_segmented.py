"""Segmented primitives (one launch over many uneven segments) against the per-segment
oracle, through the C ABI on device pointers. Integer and ordering results bit-exact; fp32
sums and prefixes within 1e-5 and fp64 within 1e-12 relative error of the compensated fp64
oracle (prefix errors relative to max(|prefix|, 1))."""
from __future__ import annotations

import numpy as np
import pytest

import cases
from cases import F32_TOL, F64_TOL

pytestmark = pytest.mark.gpu

DTYPES = {"f32": np.float32, "f64": np.float64, "i32": np.int32, "i64": np.int64,
          "u32": np.uint32, "u64": np.uint64}
LAYOUTS = cases.segment_layouts()


def make(ox, t: str, n: int, seed: int = 3) -> np.ndarray:
    if t == "f32":
        return ox.gen("f32_unit", seed, n)
    if t == "f64":
        return ox.gen("f64_unit", seed, n)
    if t == "i32":
        return ox.gen("i32_pm1000", seed, n)
    if t == "i64":
        return ox.gen("i64_full", seed, n)
    if t == "u32":
        return ox.gen("u32_full", seed, n)
    return ox.gen_u64(seed, n)


def tol(t: str) -> float:
    return F32_TOL if t == "f32" else F64_TOL


def seg_reduce(lib, px, dev, t, x, off):
    S = off.size - 1
    d, o = dev.put(x), dev.put(off)
    r = dev.empty(S * x.itemsize)
    lib.parallax_segmented_reduce(px.builtin(f"reduce:sum:{t}"), d.data_ptr(), x.size,
                                  o.data_ptr(), S, r.data_ptr())
    px.check("parallax_segmented_reduce")
    return dev.get(r, x.dtype, S)


def seg_exscan(lib, px, dev, t, x, off, init):
    S = off.size - 1
    d, o = dev.put(x), dev.put(off)
    out = dev.empty(x.nbytes)
    iv = np.array([init], dtype=x.dtype)
    lib.parallax_segmented_exclusive_scan(px.builtin(f"exclusive_scan:{t}"), d.data_ptr(),
                                          out.data_ptr(), x.size, o.data_ptr(), S,
                                          iv.ctypes.data)
    px.check("parallax_segmented_exclusive_scan")
    return dev.get(out, x.dtype, x.size)


def check_reduce(t, got, want):
    if t in ("f32", "f64"):
        assert cases_rel(got, want) <= tol(t)
    else:
        assert np.array_equal(got, want)


def cases_rel(got, want) -> float:
    g = np.asarray(got, np.float64)
    w = np.asarray(want, np.float64)
    den = np.maximum(np.abs(w), 1.0)
    return float(np.max(np.abs(g - w) / den)) if g.size else 0.0


@pytest.mark.parametrize("t", list(DTYPES))
@pytest.mark.parametrize("layout", list(LAYOUTS))
def test_segmented_reduce(lib, px, ox, dev, t, layout):
    off = LAYOUTS[layout]
    x = make(ox, t, int(off[-1]))
    got = seg_reduce(lib, px, dev, t, x, off)
    check_reduce(t, got, ox.seg_sum(x, off))


@pytest.mark.parametrize("t", list(DTYPES))
@pytest.mark.parametrize("layout", list(LAYOUTS))
def test_segmented_exclusive_scan(lib, px, ox, dev, t, layout):
    off = LAYOUTS[layout]
    x = make(ox, t, int(off[-1]))
    init = 2.5 if t in ("f32", "f64") else 7
    got = seg_exscan(lib, px, dev, t, x, off, init)
    want = ox.seg_exscan(x, off, init)
    if t in ("f32", "f64"):
        assert cases_rel(got, want) <= tol(t)
    else:
        assert np.array_equal(got, want)


PREDS = {"f32": ("gt", 0.5), "f64": ("le", 0.25), "i32": ("lt", 0), "i64": ("gt", 0),
         "u32": ("gt", 1 << 31), "u64": ("ne", 12345)}
PK = {"gt": 1, "ge": 2, "lt": 3, "le": 4, "eq": 5, "ne": 6}


@pytest.mark.parametrize("remove", [False, True])
@pytest.mark.parametrize("t", list(DTYPES))
@pytest.mark.parametrize("layout", list(LAYOUTS))
def test_segmented_copy_if(lib, px, ox, dev, t, layout, remove):
    off = LAYOUTS[layout]
    S = off.size - 1
    x = make(ox, t, int(off[-1]))
    pk, c = PREDS[t]
    spec = f"{'remove_if' if remove else 'copy_if'}:{t}:{pk}:{c}"
    d, o = dev.put(x), dev.put(off)
    out = dev.put(np.full(x.nbytes, 0xAB, dtype=np.uint8)) if x.size else dev.empty(8)
    cnt = dev.empty(max(S, 1) * 8)
    cnt.fill_(0xFF)
    dev.torch.cuda.synchronize()  # the runtime works on its own stream
    lib.parallax_segmented_copy_if(px.builtin(spec), d.data_ptr(), out.data_ptr(), x.size,
                                   o.data_ptr(), S, cnt.data_ptr())
    px.check("parallax_segmented_copy_if")
    got = dev.get(out, x.dtype, x.size)
    counts = dev.get(cnt, np.uint64, S)
    kept, want_counts = ox.seg_copy_if(x, off, PK[pk], c, remove=remove)
    assert np.array_equal(counts, want_counts)
    for s in range(S):
        a = int(off[s])
        k = int(want_counts[s])
        assert np.array_equal(got[a:a + k], kept[s]), f"segment {s}"


@pytest.mark.parametrize("op", ["max", "min"])
@pytest.mark.parametrize("t", list(DTYPES))
@pytest.mark.parametrize("layout", list(LAYOUTS))
def test_segmented_reduce_max_min(lib, px, ox, dev, t, layout, op):
    off = LAYOUTS[layout]
    S = off.size - 1
    x = make(ox, t, int(off[-1]), seed=13)
    d, o = dev.put(x), dev.put(off)
    r = dev.empty(max(S, 1) * x.itemsize)
    lib.parallax_segmented_reduce(px.builtin(f"reduce:{op}:{t}"), d.data_ptr(), x.size,
                                  o.data_ptr(), S, r.data_ptr())
    px.check("segmented max/min")
    got = dev.get(r, x.dtype, S)
    for s_ in range(S):
        a, b = int(off[s_]), int(off[s_ + 1])
        want = ox.reduce_minmax(x[a:b], op == "max") if b > a else x.dtype.type(0)
        assert got[s_] == want, (s_, got[s_], want)


@pytest.mark.parametrize("t", list(DTYPES))
@pytest.mark.parametrize("layout", list(LAYOUTS))
def test_segmented_inclusive_scan(lib, px, ox, dev, t, layout):
    off = LAYOUTS[layout]
    x = make(ox, t, int(off[-1]), seed=14)
    d, o = dev.put(x), dev.put(off)
    out = dev.empty(x.nbytes)
    lib.parallax_segmented_inclusive_scan(px.builtin(f"scan:{t}"), d.data_ptr(), out.data_ptr(),
                                          x.size, o.data_ptr(), off.size - 1)
    px.check("segmented inclusive scan")
    got = dev.get(out, x.dtype, x.size)
    fp = t in ("f32", "f64")
    want = np.zeros(x.size, np.float64 if fp else x.dtype)
    for s_ in range(off.size - 1):
        a, b = int(off[s_]), int(off[s_ + 1])
        if b > a:
            want[a:b] = ox.scan(x[a:b])
    if fp:
        assert cases_rel(got, want) <= tol(t)
    else:
        assert np.array_equal(got, want)


def seg_compact(lib, px, dev, fn, spec, x, off):
    S = off.size - 1
    d, o = dev.put(x), dev.put(off)
    out = dev.put(np.full(x.nbytes, 0xAB, dtype=np.uint8)) if x.size else dev.empty(8)
    cnt = dev.empty(max(S, 1) * 8)
    cnt.fill_(0xFF)
    dev.torch.cuda.synchronize()
    getattr(lib, fn)(px.builtin(spec), d.data_ptr(), out.data_ptr(), x.size, o.data_ptr(), S,
                     cnt.data_ptr())
    px.check(fn)
    return dev.get(out, x.dtype, x.size), dev.get(cnt, np.uint64, S)


@pytest.mark.parametrize("t,m,r", [("i32", 3, 0), ("i32", 7, -2), ("u32", 5, 1), ("i64", 3, 0),
                                   ("u64", 10, 3)])
@pytest.mark.parametrize("layout", ["tile_edges", "big_and_small", "lognormal", "mixed_empty"])
def test_segmented_copy_if_modulo(lib, px, ox, dev, t, m, r, layout):
    off = LAYOUTS[layout]
    x = make(ox, t, int(off[-1]), seed=15)
    got, counts = seg_compact(lib, px, dev, "parallax_segmented_copy_if",
                              f"copy_if:{t}:mod:{m}:{r}", x, off)
    for s_ in range(off.size - 1):
        a, b = int(off[s_]), int(off[s_ + 1])
        want, wk = ox.compact(x[a:b], ox.COPY_IF, ox.P_MOD, 0.0, m, r)
        assert counts[s_] == wk and np.array_equal(got[a:a + wk], want[:wk]), s_


@pytest.mark.parametrize("t", list(DTYPES))
@pytest.mark.parametrize("layout", list(LAYOUTS))
def test_segmented_partition(lib, px, ox, dev, t, layout):
    off = LAYOUTS[layout]
    x = make(ox, t, int(off[-1]), seed=16)
    pk, c = PREDS[t]
    got, counts = seg_compact(lib, px, dev, "parallax_segmented_partition",
                              f"partition:{t}:{pk}:{c}", x, off)
    for s_ in range(off.size - 1):
        a, b = int(off[s_]), int(off[s_ + 1])
        want, wk = ox.compact(x[a:b], ox.PARTITION, PK[pk], c)
        assert counts[s_] == wk, s_
        assert np.array_equal(got[a:b], want), s_


@pytest.mark.parametrize("t", list(DTYPES))
@pytest.mark.parametrize("layout", list(LAYOUTS))
def test_segmented_unique(lib, px, ox, dev, t, layout):
    off = LAYOUTS[layout]
    x = make(ox, t, int(off[-1]), seed=17)
    # runs of equal values inside every segment (sorted per segment, values coarsened)
    x = (x // x.dtype.type(97)) if t not in ("f32", "f64") else np.round(x * 40).astype(x.dtype)
    x = ox.seg_sort(x, off)
    got, counts = seg_compact(lib, px, dev, "parallax_segmented_unique", f"unique:{t}", x, off)
    for s_ in range(off.size - 1):
        a, b = int(off[s_]), int(off[s_ + 1])
        want, wk = ox.compact(x[a:b], ox.UNIQUE)
        assert counts[s_] == wk and np.array_equal(got[a:a + wk], want[:wk]), s_


@pytest.mark.parametrize("shift", [1, 2, 3])
def test_segmented_unaligned_arrays(lib, px, ox, dev, shift):
    """Input and output arrays that start off a 16-byte boundary (and at different phases
    from each other): tiles are staged at their own phase and stored element by element
    when the phases differ."""
    off = LAYOUTS["lognormal"]
    n = int(off[-1])
    x = make(ox, "i32", n, seed=18)
    buf = dev.put(np.concatenate([np.zeros(shift, np.int32), x]))
    o = dev.put(off)
    out = dev.empty((n + 4) * 4)
    lib.parallax_segmented_inclusive_scan(px.builtin("scan:i32"), buf.data_ptr() + 4 * shift,
                                          out.data_ptr() + 4, n, o.data_ptr(), off.size - 1)
    px.check("unaligned segmented scan")
    got = out[4: 4 + n * 4].cpu().numpy().view(np.int32)
    want = np.concatenate([ox.scan(x[int(off[i]):int(off[i + 1])]) for i in range(off.size - 1)
                           if off[i + 1] > off[i]])
    assert np.array_equal(got, want)
    r = dev.empty((off.size - 1) * 4)
    lib.parallax_segmented_reduce(px.builtin("reduce:sum:i32"), buf.data_ptr() + 4 * shift, n,
                                  o.data_ptr(), off.size - 1, r.data_ptr())
    px.check("unaligned segmented reduce")
    assert np.array_equal(dev.get(r, np.int32, off.size - 1), ox.seg_sum(x, off))


@pytest.mark.parametrize("path", ["auto", "radix", "merge"])
@pytest.mark.parametrize("t", list(DTYPES))
@pytest.mark.parametrize("layout", list(LAYOUTS))
def test_segmented_sort(lib, px, ox, dev, t, layout, path, monkeypatch):
    """Both segmented sort paths (one-sweep radix over segment-local tiles, and tile sort +
    per-segment merge passes; `auto` picks radix when the mean segment spans a radix tile)
    return the oracle's bytes on every layout."""
    if path != "auto":
        monkeypatch.setenv("PARALLAX_SORT", path)
    off = LAYOUTS[layout]
    x = make(ox, t, int(off[-1]))
    d, o = dev.put(x), dev.put(off)
    lib.parallax_segmented_sort(px.builtin(f"sort:{t}"), d.data_ptr(), x.size, o.data_ptr(),
                                off.size - 1)
    px.check("parallax_segmented_sort")
    got = dev.get(d, x.dtype, x.size)
    assert np.array_equal(got.view(np.uint8), ox.seg_sort(x, off).view(np.uint8))


@pytest.mark.parametrize("values", ["index", "random"])
@pytest.mark.parametrize("layout", ["lognormal", "tile_edges", "big_and_small", "ones"])
def test_segmented_sort_kv_stable(lib, px, ox, dev, values, layout):
    """sort_kv:u32 records (key << 32 | value) sort stably by key inside each segment: equal
    keys keep their input order whatever their values (random values would be reordered by
    a sort of the whole 64-bit records)."""
    off = LAYOUTS[layout]
    n = int(off[-1])
    keys = (ox.gen("u32_full", 5, n) % 97).astype(np.uint64)
    vals = (np.arange(n, dtype=np.uint64) if values == "index"
            else ox.gen("u32_full", 6, n).astype(np.uint64))
    recs = (keys << np.uint64(32)) | vals
    d, o = dev.put(recs), dev.put(off)
    lib.parallax_segmented_sort(px.builtin("sort_kv:u32"), d.data_ptr(), n, o.data_ptr(),
                                off.size - 1)
    px.check("parallax_segmented_sort")
    got = dev.get(d, np.uint64, n)
    for s in range(off.size - 1):
        a, b = int(off[s]), int(off[s + 1])
        seg = recs[a:b]
        order = np.argsort(seg >> np.uint64(32), kind="stable")
        assert np.array_equal(got[a:b], seg[order])


def test_segmented_sort_special_floats(lib, px, ox, dev):
    vals = np.array([np.nan, -np.inf, np.inf, -0.0, 0.0, 1.5, -1.5, -np.nan], np.float32)
    x = np.tile(vals, 700)
    off = cases.offsets_of([8, 1000, 0, 3000, 1592])
    d, o = dev.put(x), dev.put(off)
    lib.parallax_segmented_sort(px.builtin("sort:f32"), d.data_ptr(), x.size, o.data_ptr(),
                                off.size - 1)
    px.check("parallax_segmented_sort")
    got = dev.get(d, np.float32, x.size)
    assert np.array_equal(got.view(np.uint32), ox.seg_sort(x, off).view(np.uint32))


def test_replay_sees_new_data(lib, px, ox, dev):
    """The second call with the same arguments replays the captured launch sequence; it
    must read the buffers' current contents and a fresh look-back epoch each time."""
    off = LAYOUTS["lognormal"]
    n = int(off[-1])
    d, o = dev.put(make(ox, "i32", n, 1)), dev.put(off)
    out = dev.empty(n * 4)
    h = px.builtin("exclusive_scan:i32")
    iv = np.array([0], np.int32)
    for seed in range(1, 6):
        x = make(ox, "i32", n, seed)
        d.copy_(dev.put(x))
        dev.torch.cuda.synchronize()  # the runtime works on its own stream
        lib.parallax_segmented_exclusive_scan(h, d.data_ptr(), out.data_ptr(), n, o.data_ptr(),
                                              off.size - 1, iv.ctypes.data)
        px.check("replay")
        assert np.array_equal(dev.get(out, np.int32, n), ox.seg_exscan(x, off, 0))


def test_many_calls_with_different_shapes(lib, px, ox, dev):
    """Alternating segment counts reuse the shared work-list buffers: results stay exact."""
    h = px.builtin("reduce:sum:i64")
    for i, layout in enumerate(list(LAYOUTS) * 2):
        off = LAYOUTS[layout]
        x = make(ox, "i64", int(off[-1]), seed=20 + i)
        got = seg_reduce(lib, px, dev, "i64", x, off)
        assert np.array_equal(got, ox.seg_sum(x, off)), layout
    del h


def test_device_resident_arena_operands(lib, px, ox):
    from helpers import Arena
    arena = Arena(lib)
    try:
        off = LAYOUTS["tile_edges"]
        x = make(ox, "u32", int(off[-1]))
        data, offs = arena.array(x), arena.array(off)
        for a in (data, offs):
            assert lib.parallax_arena_set_residency(a.ctypes.data, px.DEVICE_RESIDENT) == px.OK
            assert lib.parallax_arena_sync_to_device(a.ctypes.data, a.nbytes) == px.OK
        lib.parallax_segmented_sort(px.builtin("sort:u32"), data.ctypes.data, x.size,
                                    offs.ctypes.data, off.size - 1)
        px.check("segmented sort on the arena")
        assert np.array_equal(data, x)  # host mirror untouched until synced
        assert lib.parallax_arena_sync_to_host(data.ctypes.data, data.nbytes) == px.OK
        assert np.array_equal(data, ox.seg_sort(x, off))
        # a coherent block is refused (its host mirror would be stale)
        lib.parallax_arena_set_residency(data.ctypes.data, px.COHERENT)
        st = lib.parallax_segmented_sort(px.builtin("sort:u32"), data.ctypes.data, x.size,
                                         offs.ctypes.data, off.size - 1)
        assert st == px.ERR_INVALID_ARGUMENT
        lib.parallax_clear_error()
        lib.parallax_arena_set_residency(offs.ctypes.data, px.COHERENT)
    finally:
        arena.free()


def test_bad_offsets_are_reported(lib, px, dev):
    x = dev.put(np.arange(100, dtype=np.float32))
    r = dev.empty(16)
    for bad in ([0, 50, 40], [0, 60, 101]):
        off = dev.put(np.array(bad, np.uint64))
        st = lib.parallax_segmented_reduce(px.builtin("reduce:sum:f32"), x.data_ptr(), 100,
                                           off.data_ptr(), 2, r.data_ptr())
        assert st == px.ERR_INVALID_ARGUMENT
        lib.parallax_clear_error()
        st = lib.parallax_segmented_sort(px.builtin("sort:f32"), x.data_ptr(), 100,
                                         off.data_ptr(), 2)
        assert st == px.ERR_INVALID_ARGUMENT
        lib.parallax_clear_error()


def test_rejects_host_and_coherent_operands(lib, px, ox):
    off = cases.offsets_of([3, 4])
    x = np.arange(7, dtype=np.float32)
    r = np.zeros(2, np.float32)
    st = lib.parallax_segmented_reduce(px.builtin("reduce:sum:f32"), x.ctypes.data, 7,
                                       off.ctypes.data, 2, r.ctypes.data)
    assert st == px.ERR_INVALID_ARGUMENT
    lib.parallax_clear_error()


def test_rejects_wrong_handles(lib, px, dev):
    off = dev.put(cases.offsets_of([3, 4]))
    x = dev.put(np.arange(7, dtype=np.float32))
    r = dev.empty(64)
    assert lib.parallax_segmented_reduce(px.builtin("sort:f32"), x.data_ptr(), 7,
                                         off.data_ptr(), 2, r.data_ptr()) == px.ERR_INVALID_HANDLE
    assert lib.parallax_segmented_sort(px.builtin("reduce:sum:f32"), x.data_ptr(), 7,
                                       off.data_ptr(), 2) == px.ERR_INVALID_HANDLE
    assert lib.parallax_segmented_copy_if(px.builtin("scan:f32"), x.data_ptr(),
                                          r.data_ptr(), 7, off.data_ptr(), 2,
                                          r.data_ptr()) == px.ERR_INVALID_HANDLE
    assert lib.parallax_segmented_partition(px.builtin("copy_if:f32:gt:0"), x.data_ptr(),
                                            r.data_ptr(), 7, off.data_ptr(), 2,
                                            r.data_ptr()) == px.ERR_INVALID_HANDLE
    assert lib.parallax_segmented_unique(px.builtin("copy_if:f32:gt:0"), x.data_ptr(),
                                         r.data_ptr(), 7, off.data_ptr(), 2,
                                         r.data_ptr()) == px.ERR_INVALID_HANDLE
    lib.parallax_clear_error()


def test_zero_segments_is_a_no_op(lib, px, dev):
    x = dev.put(np.arange(7, dtype=np.float32))
    off = dev.put(np.zeros(1, np.uint64))
    r = dev.empty(8)
    assert lib.parallax_segmented_reduce(px.builtin("reduce:sum:f32"), x.data_ptr(), 0,
                                         off.data_ptr(), 0, r.data_ptr()) == px.OK
    assert lib.parallax_segmented_sort(px.builtin("sort:f32"), x.data_ptr(), 0,
                                       off.data_ptr(), 0) == px.OK


_TUNE_SCRIPT = r'''
import ctypes as C, importlib.util, sys
import numpy as np, torch
spec = importlib.util.spec_from_file_location("parallax_runtime_b200", sys.argv[1])
px = importlib.util.module_from_spec(spec); spec.loader.exec_module(px)
lib = px.load()
off = np.array([0, 70000, 70001, 200000], np.uint64)
x = torch.ones(200000, dtype=torch.float32, device="cuda")
o = torch.from_numpy(off.view(np.uint8)).cuda()
r = torch.zeros(3, dtype=torch.float32, device="cuda")
torch.cuda.synchronize()
lib.parallax_segmented_reduce(px.builtin("reduce:sum:f32"), x.data_ptr(), 200000, o.data_ptr(), 3,
                              r.data_ptr())
px.check("tuned reduce")
assert r.cpu().tolist() == [70000.0, 1.0, 129999.0], r
'''


def test_tuner_cache_is_written_and_reused(tmp_path):
    """The autotuner times the tile candidates once per (op, type, size bucket), stores the
    choice in PARALLAX_TUNE_CACHE, and a later process reuses it without timing."""
    import os
    import subprocess
    import sys

    from conftest import ROOT
    cache = tmp_path / "tune.txt"
    script = tmp_path / "run.py"
    script.write_text(_TUNE_SCRIPT)
    env = dict(os.environ, PARALLAX_TUNE_CACHE=str(cache), PARALLAX_DEBUG="1")
    env.pop("PARALLAX_TUNE", None)
    pkg = str(ROOT / "parallax-runtime_b200" / "__init__.py")
    r1 = subprocess.run([sys.executable, str(script), pkg], env=env, capture_output=True,
                        text=True, timeout=300)
    assert r1.returncode == 0, r1.stderr[-2000:]
    assert "tuned segmented op 0" in r1.stderr
    entries = [ln.split() for ln in cache.read_text().splitlines() if ln.strip()]
    assert entries and all(len(e) == 5 and e[3] in ("256", "512") and e[4] in ("3", "7")
                           for e in entries)
    r2 = subprocess.run([sys.executable, str(script), pkg], env=env, capture_output=True,
                        text=True, timeout=300)
    assert r2.returncode == 0, r2.stderr[-2000:]
    assert "tuned segmented op" not in r2.stderr
