"""The reference's own stdpar.hpp linked against this runtime, on a B200.

oracle/stdpar_driver.cpp calls the reference's parallax:: algorithms (its unmodified
include/parallax/stdpar.hpp, compiled by oracle/Makefile where the reference tree is
present) on seeded inputs. Built twice: `stdpar_driver_gpu` links libparallax-runtime.so
(fixed funnels hit the built-in sm_100a kernels, functor funnels the sm_100a images the
driver registers under their funnel keys), `stdpar_driver_host` links an ABI whose lookups
all miss, so every call runs the reference's host fallback. Each call's result is compared
between the two runs: integer and element-wise results bit-exact, sorts as values (the
host's std::sort may order -0.0 and +0.0 either way; the device gives the IEEE total order,
checked byte-exact against the oracle), floating-point sums and prefixes against the
compensated oracle within 1e-5 (fp32) / 1e-12 (fp64) (the host fallback is a left fold),
partition against the stable oracle (the host fallback, std::partition, is unstable).
Every device-side call must have launched runtime kernels; the host run launches none.

A third build, `stdpar_driver_heap`, also links the whole-heap capture shim
(lib/libparallax-heap.a, reference src/memory/heap_capture.cpp): every std::vector of the
program lives in the runtime's heap pool, the arena adopts the pool (zero-copy), the funnels
find their data in the arena and call the runtime on it in place, and a transform chases
pointers stored in heap records. Its results must match the host run the same way.

The count_if and transform_reduce transforms are registered as images that also export
their element function (LTO-IR), so each of those funnels must run as one fused launch.
"""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

from cases import F32_TOL, F64_TOL

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
REF = ROOT / "oracle" / "_ref"
IMAGES = Path(__file__).resolve().parent / "images" / "_build"
SIZES = (1, 1000, 300007)


def parse(path: Path) -> dict[str, tuple[int, int, bytes]]:
    raw = path.read_bytes()
    out, i = {}, 0
    while i < len(raw):
        j = raw.index(b"\0", i)
        name = raw[i:j].decode()
        launches, scalar, nbytes = np.frombuffer(raw[j + 1: j + 25], np.uint64)
        data = raw[j + 25: j + 25 + int(nbytes)]
        out[name] = (int(launches), int(scalar), data)
        i = j + 25 + int(nbytes)
    return out


@pytest.fixture(scope="module")
def runs(tmp_path_factory):
    exe = {k: REF / f"stdpar_driver_{k}" for k in ("gpu", "heap", "host")}
    if not all(p.exists() for p in exe.values()):
        pytest.skip("stdpar drivers not built (oracle/Makefile needs the reference's headers)")
    d = tmp_path_factory.mktemp("stdpar")
    res = {}
    for k, p in exe.items():
        out = d / f"{k}.bin"
        env = dict(os.environ, PARALLAX_HEAP_POOL="16384")
        r = subprocess.run([str(p), str(IMAGES), str(out)], capture_output=True, text=True,
                           timeout=600, env=env)
        assert r.returncode == 0, f"{p.name} failed ({r.returncode}):\n{r.stdout}\n{r.stderr}"
        res[k] = parse(out)
    # the pointer-chasing transform runs only where stored heap pointers reach the device
    gather = {k for k in res["host"] if k.startswith("transform_gather")}
    assert res["gpu"].keys() == res["host"].keys() - gather
    assert res["heap"].keys() == res["host"].keys()
    return res


BUILDS = ("gpu", "heap")


def inputs(ox, n):
    f32 = ox.gen("f32_unit", 21, n)
    f64 = ox.gen("f64_unit", 22, n)
    i32 = ox.gen("i32_pm1000", 23, n)
    i64 = ox.gen("i64_full", 24, n)
    return f32, f64, i32, i64


def arr(rec, dtype):
    return np.frombuffer(rec[2], dtype)


def scalar(rec, dtype):
    """The record's scalar: the value's bytes in the low bytes of a uint64."""
    v = np.array([rec[1]], np.uint64)
    if np.dtype(dtype).itemsize == 8:
        return v.view(dtype)[0]
    return v.astype(np.uint32).view(dtype)[0]


# calls the runtime may finish without a launch: one-element scan in place and sort
NO_LAUNCH_AT_1 = {"inclusive_scan_f32", "inclusive_scan_i64", "sort_u32", "sort_f32"}


@pytest.mark.parametrize("build", BUILDS)
@pytest.mark.parametrize("n", SIZES)
def test_every_call_went_through_the_runtime(runs, n, build):
    for name, (launches, _, _) in runs[build].items():
        base, size = name.split("@")
        if int(size) != n:
            continue
        assert runs["host"][name][0] == 0
        if (n == 1 and base in NO_LAUNCH_AT_1) or base == "heap_capture":
            continue
        assert launches > 0, f"{name}: no runtime kernel launched (the funnel fell back)"


@pytest.mark.parametrize("build", BUILDS)
@pytest.mark.parametrize("n", SIZES)
def test_reduce_and_scans(runs, build, ox, n):
    g, h = runs[build], runs["host"]
    f32, f64, i32, i64 = inputs(ox, n)
    s = f"@{n}"
    got = scalar(g["reduce_f32" + s], np.float32)
    want = ox.reduce_sum(f32)
    assert abs(float(got) - want) <= F32_TOL * abs(want)
    got = scalar(g["reduce_f64" + s], np.float64)
    assert abs(float(got) - ox.reduce_sum(f64)) <= F64_TOL * abs(ox.reduce_sum(f64))
    assert scalar(g["reduce_i32" + s], np.int32) == scalar(h["reduce_i32" + s], np.int32) \
        == ox.reduce_sum(i32)
    assert scalar(g["reduce_i64" + s], np.int64) == ox.reduce_sum(i64)
    assert ox.max_rel_err(arr(g["inclusive_scan_f32" + s], np.float32), ox.scan(f32)) <= F32_TOL
    assert np.array_equal(arr(g["inclusive_scan_i64" + s], np.int64), ox.scan(i64))
    assert np.array_equal(arr(g["exclusive_scan_i32" + s], np.int32),
                          arr(h["exclusive_scan_i32" + s], np.int32))
    assert np.array_equal(arr(g["exclusive_scan_i32" + s], np.int32),
                          ox.scan(i32, exclusive=True, init=5))
    ex = arr(g["exclusive_scan_f64" + s], np.float64)
    want = ox.scan(f64, exclusive=True, init=0.25)
    assert ox.max_rel_err(ex, want) <= F64_TOL


@pytest.mark.parametrize("build", BUILDS)
@pytest.mark.parametrize("n", SIZES)
def test_sort_and_unique(runs, build, ox, n):
    g, h = runs[build], runs["host"]
    s = f"@{n}"
    got = arr(g["sort_u32" + s], np.uint32)
    assert np.array_equal(got, arr(h["sort_u32" + s], np.uint32))
    assert np.array_equal(got, np.sort(ox.gen("u32_full", 25, n)))
    f = ox.gen("f32_unit", 26, n) * np.float32(2) - np.float32(1)
    f[: n // 50] = f[n // 2: n // 2 + n // 50]
    if n > 3:
        f[1], f[3] = np.float32(0.0), np.float32(-0.0)
    got = arr(g["sort_f32" + s], np.float32)
    assert np.array_equal(got, arr(h["sort_f32" + s], np.float32))  # as values
    assert np.array_equal(got.view(np.uint32), ox.sort(f).view(np.uint32))  # total order
    k = g["unique_i32" + s][1]
    assert k == h["unique_i32" + s][1]
    assert np.array_equal(arr(g["unique_i32" + s], np.int32), arr(h["unique_i32" + s], np.int32))


@pytest.mark.parametrize("build", BUILDS)
@pytest.mark.parametrize("n", SIZES)
def test_compaction_with_registered_predicates(runs, build, ox, n):
    g, h = runs[build], runs["host"]
    s = f"@{n}"
    for name in ("copy_if_mod3_i32", "remove_if_mod3_i32"):
        assert g[name + s][1] == h[name + s][1], name
        assert np.array_equal(arr(g[name + s], np.int32), arr(h[name + s], np.int32)), name
    x = ox.gen("i32_pm1000", 23, n)
    want, wk = ox.compact(x, ox.PARTITION, ox.P_LT, 0.0)
    gp, hp = g["partition_neg_i32" + s], h["partition_neg_i32" + s]
    assert gp[1] == hp[1] == wk
    assert np.array_equal(arr(gp, np.int32), want)  # stable
    hv = arr(hp, np.int32)  # std::partition: same split, any order within each side
    assert np.all(hv[:wk] < 0) and np.all(hv[wk:] >= 0)
    assert np.array_equal(np.sort(hv), np.sort(x))


@pytest.mark.parametrize("build", BUILDS)
@pytest.mark.parametrize("n", SIZES)
def test_element_wise_funnels_with_registered_images(runs, build, n):
    g, h = runs[build], runs["host"]
    s = f"@{n}"
    for name, dt in (("for_each_affine_f32", np.float32), ("for_each_default_f32", np.float32),
                     ("transform_half_i32", np.float64)):
        assert np.array_equal(arr(g[name + s], dt).view(np.uint8),
                              arr(h[name + s], dt).view(np.uint8)), name
    assert g["count_if_gt_half_f32" + s][1] == h["count_if_gt_half_f32" + s][1]
    # sums of x * 0.5 over int32 are exact in fp64: the fused pass gives the host's bits
    assert g["transform_reduce_half_i32" + s][1] == h["transform_reduce_half_i32" + s][1]
    # both transforms export their element function: each funnel ran as ONE fused pass
    # (transform + reduce in one kernel) instead of a transform kernel and a reduce kernel
    for name in ("count_if_gt_half_f32", "transform_reduce_half_i32"):
        assert g[name + s][0] == 1, f"{name}: {g[name + s][0]} launches, not one fused pass"


@pytest.mark.parametrize("n", SIZES)
def test_whole_heap_capture(runs, n):
    """Under capture the program's vectors are heap-pool memory that the arena adopted
    (parallax_heap_contains and parallax_arena_contains both 1); without it, neither. The
    transform over heap records that store pointers into another heap array gives the host
    fallback's bytes (relocation of stored heap pointers)."""
    s = f"@{n}"
    assert runs["heap"]["heap_capture" + s][1] == 3
    assert runs["gpu"]["heap_capture" + s][1] == 0
    assert runs["host"]["heap_capture" + s][1] == 0
    g, h = runs["heap"]["transform_gather_f32" + s], runs["host"]["transform_gather_f32" + s]
    assert g[0] > 0
    assert g[2] == h[2]

