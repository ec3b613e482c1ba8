"""Bounded in-kernel waits on a B200, without a GPU fault: a look-back whose predecessor
never publishes (a tile launched as tile 1 of a fresh epoch, so nothing ever sets the flag
it polls) gives up after its poll limit, the kernel returns, the call reports
PARALLAX_ERR_DEVICE_SPIN, and the context stays usable for the next call. The reference's
fence waits have no limit (src/kernel/kernel_launcher.cpp:438-443)."""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent


@pytest.mark.parametrize("polls", [1, 256, 100000])
def test_unsatisfiable_wait_gives_up_and_the_context_survives(lib, px, ox, dev, polls):
    st = lib.parallax_check_bounded_wait(polls)
    assert st == px.ERR_DEVICE_SPIN
    assert lib.parallax_last_error() == px.ERR_DEVICE_SPIN
    lib.parallax_clear_error()
    # the next call on the same thread and stream works and is correct
    x = ox.gen("i32_pm1000", 31, 1 << 20)
    d = dev.put(x)
    dev.torch.cuda.synchronize()
    h = px.builtin("scan:i32")
    lib.parallax_scan(h, h, d.data_ptr(), x.size, 4)
    px.check("scan after a wait gave up")
    assert np.array_equal(dev.get(d, np.int32, x.size), ox.scan(x))


def test_wait_limit_knob_keeps_normal_calls_correct(tmp_path):
    """PARALLAX_WAIT_LIMIT lowers every look-back's poll limit; at a limit that real
    predecessors meet, large scans still complete with exact results."""
    code = f"""
import sys, ctypes as C, numpy as np
sys.path.insert(0, {str(ROOT)!r}); sys.path.insert(0, {str(ROOT / 'tests')!r})
import conftest, oracle
px = conftest._load_pkg(); lib = px.load(); d = conftest.Dev()
x = oracle.gen("i64_full", 32, (1 << 24) + 5)
t = d.put(x); d.torch.cuda.synchronize()
h = px.builtin("scan:i64")
lib.parallax_scan(h, h, t.data_ptr(), x.size, 8); px.check("scan")
assert np.array_equal(d.get(t, np.int64, x.size), oracle.scan(x))
assert lib.parallax_check_bounded_wait(4096) == px.ERR_DEVICE_SPIN
print("ok")
"""
    env = dict(os.environ, PARALLAX_WAIT_LIMIT="200000")
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr
