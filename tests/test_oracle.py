"""The CPU oracle, pinned against the reference's own outputs (golden vectors from its
stdpar.hpp host fallbacks) and the reference unit tests' known answers. CPU only."""
from __future__ import annotations

import numpy as np
import pytest

import cases
from cases import F32_TOL, F64_TOL, SIZES, golden, same_as_golden

pytestmark = []


@pytest.mark.parametrize("n", SIZES)
def test_reduce_matches_reference(ox, n):
    x = cases.inputs(n)
    g = golden()
    assert ox.reduce_sum(x["i32"]) == g[f"reduce_i32_{n}"][0]
    assert ox.reduce_sum(x["i64"]) == g[f"reduce_i64_{n}"][0]
    # the reference's fp32 left fold is itself inexact; at these sizes it is within 1e-5
    want = float(g[f"reduce_f32_{n}"][0])
    assert abs(ox.reduce_sum(x["f32"]) - want) <= F32_TOL * abs(want)
    want = float(g[f"reduce_f64_{n}"][0])
    assert abs(ox.reduce_sum(x["f64"]) - want) <= F64_TOL * abs(want)


@pytest.mark.parametrize("n", SIZES)
def test_scans_match_reference(ox, n):
    x = cases.inputs(n)
    for t in ("i32", "i64"):
        assert same_as_golden(f"inclusive_scan_{t}_{n}", ox.scan(x[t]))
        assert same_as_golden(f"exclusive_scan_{t}_{n}", ox.scan(x[t], exclusive=True, init=7))
    if n <= 5000:
        ref = golden()[f"inclusive_scan_f32_{n}"]
        assert ox.max_rel_err(ref, ox.scan(x["f32"])) <= F32_TOL


@pytest.mark.parametrize("n", SIZES)
def test_sort_matches_reference(ox, n):
    x = cases.inputs(n)
    assert same_as_golden(f"sort_u32_{n}", ox.sort(x["u32"]))
    assert same_as_golden(f"sort_i32_{n}", ox.sort(x["i32"]))
    if n <= 5000:
        assert np.array_equal(ox.sort(x["f32"]), golden()[f"sort_f32_{n}"])


@pytest.mark.parametrize("n", SIZES)
def test_compaction_matches_reference(ox, n):
    x = cases.inputs(n)
    i32 = x["i32"]
    out, k = ox.compact(i32, ox.COPY_IF, ox.P_MOD, m=3, r=0)
    assert same_as_golden(f"copy_if_mod3_i32_{n}", out[:k])
    out, k = ox.compact(i32, ox.REMOVE_IF, ox.P_MOD, m=3, r=0)
    assert same_as_golden(f"remove_if_mod3_i32_{n}", out[:k])
    u = cases.unique_input(i32)
    out, k = ox.compact(u, ox.UNIQUE)
    assert same_as_golden(f"unique_i32_{n}", out[:k])
    out, k = ox.compact(x["f32"], ox.COPY_IF, ox.P_GT, c=0.5)
    if n <= 5000:
        assert same_as_golden(f"copy_if_gthalf_f32_{n}", out[:k])


@pytest.mark.parametrize("n", [n for n in SIZES if n <= 5000])
def test_partition_matches_reference_as_sets(ox, n):
    # std::partition (the reference fallback) is not stable: compare the two halves as
    # multisets; the oracle's own order is the stable one.
    i32 = cases.inputs(n)["i32"]
    g = golden()
    want, wk = g[f"partition_neg_i32_{n}"], int(g[f"partition_neg_i32_{n}_k"][0])
    out, k = ox.compact(i32, ox.PARTITION, ox.P_LT, c=0)
    assert k == wk
    assert np.array_equal(np.sort(out[:k]), np.sort(want[:k]))
    assert np.array_equal(np.sort(out[k:]), np.sort(want[k:]))
    assert np.array_equal(out[:k], i32[i32 < 0]) and np.array_equal(out[k:], i32[i32 >= 0])


def test_known_answers(ox):
    x, want = cases.kat_reduce()
    assert ox.reduce_sum(x) == want
    x, want = cases.kat_scan()
    assert np.array_equal(ox.scan(x).astype(np.float32), want)
    x = cases.kat_sort()
    y = ox.sort(x)
    assert np.all(np.diff(y) >= 0) and y.astype(np.uint64).sum() == x.astype(np.uint64).sum()
    x, wk, want = cases.kat_copy_if()
    out, k = ox.compact(x, ox.COPY_IF, ox.P_GT, c=0.5)
    assert k == wk and np.array_equal(out[:k], want)


def test_generators_are_counter_based(ox):
    a = ox.gen_u64(5, 100)
    b = ox.gen_u64(5, 60, start=40)
    assert np.array_equal(a[40:], b)
    f = ox.gen("f32_unit", 3, 1000)
    assert f.min() >= 0 and f.max() < 1
    i = ox.gen("i32_pm1000", 3, 10000)
    assert i.min() >= -1000 and i.max() <= 1000


def test_oracle_against_compiled_reference(ox):
    ref = ox.ref()
    if ref is None:
        pytest.skip("reference CPU path not built here (golden vectors cover it)")
    import ctypes as C
    x = ox.gen("i32_pm1000", 9, 100003)
    ref.ref_reduce_i32.restype = C.c_int32
    assert ref.ref_reduce_i32(C.c_void_p(x.ctypes.data), x.size) == ox.reduce_sum(x)
    y = np.empty_like(x)
    ref.ref_inclusive_scan_i32(C.c_void_p(x.ctypes.data), C.c_void_p(y.ctypes.data), x.size)
    assert np.array_equal(y, ox.scan(x))


def test_fp32_fallback_is_not_the_fp_oracle(ox):
    # The reference's fp32 left fold stalls at 2^24 (16777216 + 1.0 == 16777216 in fp32);
    # the oracle accumulates in compensated fp64, so FP parity is judged against it.
    x = np.ones(1 << 25, np.float32)
    assert ox.reduce_sum(x) == float(1 << 25)
