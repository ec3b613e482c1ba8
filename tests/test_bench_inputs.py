"""bench.py generates its inputs without the oracle; they must be the oracle's arrays."""
from __future__ import annotations

import importlib.util

import numpy as np
import pytest

from conftest import ROOT


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.mark.parametrize("kind", ["f32_unit", "f64_unit", "i32_pm1000", "u32_full", "i64_full"])
def test_generators_match_oracle(bench, ox, kind):
    for seed, n in ((0, 1), (3, 1000), (7, (1 << 24) + 77)):
        a = bench.gen(kind, seed, n)
        b = ox.gen(kind, seed, n)
        assert a.dtype == b.dtype and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def test_splitmix_offset_start(bench, ox):
    assert np.array_equal(bench.splitmix(16, 1000, start=123), ox.gen_u64(16, 1000, start=123))


def test_step_inputs_shapes(bench):
    x = bench.make_inputs(12, 11)
    assert set(x) == {"f32", "f64", "i32", "i64", "sort_u32", "sort_f32", "part_i32", "uniq_i32"}
    assert x["sort_f32"].size == 1 << 11 and x["uniq_i32"].size == 1 << 12
    assert np.all(np.diff(x["uniq_i32"]) >= 0)
    kept = bench.expected_kept(x)
    assert kept["copy_if_i32"] == int(np.count_nonzero(x["i32"] % 3 == 0))
    assert bench.op_key("inclusive_scan_f64") == "f64" and bench.op_key("sort_f32") == "sort_f32"
    assert set(bench.make_inputs(12, 11, keys={"sort_u32"})) == {"sort_u32"}


def test_clock_summary(bench):
    """Throttle reasons and the median clock come from the sampled CSV lines; malformed and
    unavailable fields are skipped."""
    lines = [
        "0, 1965, 1965, 812.3, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "0, 1965, 1965, 990.1, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "0, 1890, 1965, 1000.2, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "garbage",
        "0, [N/A], 1965, 0, 0x0, Not Active, Not Active, Not Active, Not Active",
    ]
    c = bench.ClockSampler.summary(lines)
    assert c["samples"] == 3 and c["sm_mhz"] == 1965.0 and c["sm_max_mhz"] == 1965.0
    assert c["reasons"] == ["sw_power_cap"]
    hw = bench.ClockSampler.summary(
        ["0, 1200, 1965, 700, 0x8, Active, Not Active, Active, Not Active"])
    assert hw["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"] and hw["sm_mhz"] == 1200.0
    assert bench.ClockSampler.summary([])["samples"] == 0
