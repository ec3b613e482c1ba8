"""Heap pool and whole-heap capture, on the CPU.

The pool (csrc/heap_pool.cu) replaces the reference's src/memory/heap_pool.cpp with the same
API (include/parallax/heap_pool.h); the capture shim (heap/heap_capture.cpp, built as
lib/libparallax-heap.a) replaces src/memory/heap_capture.cpp. Everything runs in child
processes: a live pool switches the runtime's arena to its pool-backed mode, which must not
leak into the rest of a test session.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
LIB_DIR = ROOT / "parallax-runtime_b200" / "lib"

POOL_SCRIPT = r'''
import ctypes as C, random, sys
lib = C.CDLL(sys.argv[1])
vp, sz = C.c_void_p, C.c_size_t
lib.px_pool_alloc.restype = vp; lib.px_pool_alloc.argtypes = [sz, sz]
lib.px_pool_realloc.restype = vp; lib.px_pool_realloc.argtypes = [vp, sz]
lib.px_pool_free.argtypes = [vp]
lib.px_pool_usable_size.restype = sz; lib.px_pool_usable_size.argtypes = [vp]
lib.px_pool_contains.argtypes = [vp]
lib.parallax_heap_contains.argtypes = [vp]
lib.px_pool_base.restype = vp
lib.px_pool_reservation.restype = sz
lib.px_pool_high_water.restype = sz
assert lib.px_pool_base() is None and lib.px_pool_contains(16) == 0  # not yet initialized
assert lib.px_pool_init() == 1
base, res = lib.px_pool_base(), lib.px_pool_reservation()
assert base % (2 << 20) == 0 and res == 64 << 20
rng = random.Random(5)
live = {}  # ptr -> (size, byte)

def fill(p, n, b):
    C.memset(p, b, n)

def same(p, n, b):
    return C.string_at(p, n) == bytes([b]) * n

for step in range(6000):
    r = rng.random()
    if r < 0.5 or not live:
        n = rng.choice([1, 15, 16, 17, 100, 4096, 70000, rng.randint(1, 300000)])
        a = rng.choice([1, 8, 16, 64, 256, 4096])
        p = lib.px_pool_alloc(n, a)
        assert p and p % max(a, 16) == 0, (n, a)
        assert lib.px_pool_contains(p) and lib.parallax_heap_contains(p)
        assert lib.px_pool_usable_size(p) >= n
        b = rng.randrange(256)
        fill(p, n, b)
        live[p] = (n, b)
    elif r < 0.8:
        p = rng.choice(list(live))
        n, b = live.pop(p)
        assert same(p, n, b), "a block was overwritten"
        lib.px_pool_free(p)
    else:
        p = rng.choice(list(live))
        n, b = live.pop(p)
        m = rng.choice([1, n // 2 + 1, n + 1, 2 * n + 7, rng.randint(1, 400000)])
        q = lib.px_pool_realloc(p, m)
        assert q and q % 16 == 0
        assert same(q, min(n, m), b), "realloc lost contents"
        fill(q, m, b)
        live[q] = (m, b)
    if step % 500 == 0:
        assert lib.px_pool_check() == 1
# no two live blocks overlap
iv = sorted((p, p + n) for p, (n, _) in live.items())
assert all(a[1] <= b[0] for a, b in zip(iv, iv[1:]))
for p, (n, b) in live.items():
    assert same(p, n, b)
    lib.px_pool_free(p)
assert lib.px_pool_check() == 1
hw = lib.px_pool_high_water()
assert 0 < hw <= res
assert lib.px_pool_alloc(res + 1, 16) is None  # beyond the reservation
# everything was freed: the space is whole again
p = lib.px_pool_alloc(res - (1 << 20), 16)
assert p, "freed space was not coalesced"
lib.px_pool_free(p)
assert lib.px_pool_check() == 1
assert lib.px_pool_realloc(None, 100) and lib.px_pool_realloc(lib.px_pool_alloc(10, 16), 0) is None
print("ok")
'''


def test_pool_allocator_invariants():
    env = dict(os.environ, PARALLAX_HEAP_POOL="64", PARALLAX_HEAP_CHECK="1")
    r = subprocess.run([sys.executable, "-c", POOL_SCRIPT, str(LIB_DIR / "libparallax-runtime.so")],
                       env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr


def test_capture_shim_routes_the_heap_into_the_pool(tmp_path):
    exe = tmp_path / "capture_check"
    cmd = ["g++", "-std=c++17", "-O1", "-I", str(ROOT / "include"),
           str(ROOT / "tests" / "heap" / "capture_check.cpp"), str(LIB_DIR / "libparallax-heap.a"),
           "-L", str(LIB_DIR), "-lparallax-runtime", f"-Wl,-rpath,{LIB_DIR}", "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    env = dict(os.environ, PARALLAX_HEAP_POOL="1024", PARALLAX_HEAP_CHECK="0")
    r = subprocess.run([str(exe)], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.startswith("ok"), r.stdout + r.stderr
