"""The serving loop (continuous batching): every request's result is the same alone and in a
concurrent mix from many threads, and matches the oracle (integers bit-exact; fp32 within
1e-5 and fp64 within 1e-12 relative error of the compensated fp64 oracle, prefixes relative
to max(|prefix|, 1)). Also admission by memory budget, statistics and error paths."""
from __future__ import annotations

import ctypes as C
import threading

import numpy as np
import pytest

from cases import F32_TOL, F64_TOL

pytestmark = pytest.mark.gpu

SOLO = 1 << 15  # longer requests run alone: both paths are exercised
SIZES = [0, 1, 5, 1000, 4097, 30000, SOLO + 1, 70001]


def make(ox, t, n, seed):
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


class Req:
    """One request with its own device buffers and host result slot."""

    def __init__(self, px, dev, spec, x, kind, exclusive=False, init=0):
        self.spec, self.x, self.kind, self.exclusive = spec, x, kind, exclusive
        self.h = px.builtin(spec)
        self.dev = dev
        self.d_in = dev.put(x) if x.size else dev.empty(8)
        self.d_out = dev.empty(max(x.nbytes, 8)) if kind in ("exscan", "compact") else None
        self.res = np.zeros(1, np.uint64)
        self.init = np.array([init], dtype=x.dtype)
        r = px.Request()
        r.kernel = self.h
        r.input = self.d_in.data_ptr()
        r.output = self.d_out.data_ptr() if self.d_out is not None else None
        r.count = x.size
        r.init = self.init.ctypes.data
        r.result = self.res.ctypes.data
        r.flags = px.REQ_EXCLUSIVE if exclusive else 0
        self.req = r

    def output(self):
        """What the request produced: scalar result, array, or (array, kept)."""
        t = self.x.dtype
        if self.kind == "reduce":
            return self.res.view(np.uint8)[: t.itemsize].view(t)[0]
        if self.kind in ("scan", "sort"):
            return self.dev.get(self.d_in, t, self.x.size)
        if self.kind == "exscan":
            return self.dev.get(self.d_out, t, self.x.size)
        k = int(self.res[0])
        return self.dev.get(self.d_out, t, self.x.size)[:k], k


def mix(px, dev, ox, seed0=100):
    out = []
    s = seed0
    for n in SIZES:
        for t in ("f32", "f64", "i32", "i64"):
            s += 1
            out.append(Req(px, dev, f"reduce:sum:{t}", make(ox, t, n, s), "reduce"))
            out.append(Req(px, dev, f"exclusive_scan:{t}", make(ox, t, n, s + 1000), "exscan",
                           exclusive=True, init=3))
        out.append(Req(px, dev, "scan:i32", make(ox, "i32", n, s + 2000), "scan"))
        out.append(Req(px, dev, "scan:f32", make(ox, "f32", n, s + 2500), "scan"))
        out.append(Req(px, dev, "reduce:max:f64", make(ox, "f64", n, s + 3000), "reduce"))
        for t in ("u32", "f32", "i64"):
            out.append(Req(px, dev, f"sort:{t}", make(ox, t, n, s + 4000), "sort"))
        out.append(Req(px, dev, "copy_if:f32:gt:0.5", make(ox, "f32", n, s + 5000), "compact"))
        out.append(Req(px, dev, "remove_if:i32:lt:0", make(ox, "i32", n, s + 6000), "compact"))
        out.append(Req(px, dev, "copy_if:i32:mod:3:0", make(ox, "i32", n, s + 7000), "compact"))
        # same operation and type, another predicate: must never share a launch with the above
        out.append(Req(px, dev, "copy_if:i32:mod:5:1", make(ox, "i32", n, s + 7500), "compact"))
        # key-value records with random values: sorted stably by key, not by the whole record
        recs = (make(ox, "u32", n, s + 8000).astype(np.uint64) % np.uint64(37)) << np.uint64(32)
        recs |= make(ox, "u32", n, s + 8500).astype(np.uint64)
        out.append(Req(px, dev, "sort_kv:u32", recs, "sort"))
    return out


def oracle_of(ox, r: Req):
    x = r.x
    if r.kind == "reduce" and x.size == 0:
        return x.dtype.type(0)  # an empty reduce writes zeros
    if r.spec.startswith("reduce:sum"):
        return ox.reduce_sum(x)
    if r.spec.startswith("reduce:max"):
        return ox.reduce_minmax(x, True)
    if r.kind == "exscan":
        return ox.scan(x, exclusive=True, init=3)
    if r.kind == "scan":
        return ox.scan(x)
    if r.kind == "sort" and r.spec.startswith("sort_kv"):
        return x[np.argsort(x >> np.uint64(32), kind="stable")]
    if r.kind == "sort":
        return ox.sort(x)
    pk = {"gt": ox.P_GT, "lt": ox.P_LT, "mod": ox.P_MOD}[r.spec.split(":")[2]]
    if pk == ox.P_MOD:
        m, rem = (int(v) for v in r.spec.split(":")[3:5])
        out, k = ox.compact(x, ox.COPY_IF, pk, 0, m, rem)
    else:
        c = float(r.spec.split(":")[3])
        out, k = ox.compact(x, ox.REMOVE_IF if r.spec.startswith("remove") else ox.COPY_IF, pk, c)
    return out[:k], k


def rel(got, want) -> float:
    g = np.atleast_1d(np.asarray(got, np.float64))
    w = np.atleast_1d(np.asarray(want, np.float64))
    if g.size == 0:
        return 0.0
    return float(np.max(np.abs(g - w) / np.maximum(np.abs(w), 1.0)))


def same(r: Req, a, b, exact_fp=False):
    """a == b for integer work, within tolerance for floating point."""
    fp = r.x.dtype.kind == "f"
    if r.kind == "compact":
        return a[1] == b[1] and np.array_equal(a[0].view(np.uint8), b[0].view(np.uint8))
    if r.kind == "sort" or not fp or exact_fp:
        a = np.atleast_1d(np.asarray(a, dtype=r.x.dtype))
        b = np.atleast_1d(np.asarray(b, dtype=r.x.dtype))
        return np.array_equal(a.view(np.uint8), b.view(np.uint8))
    tol = F32_TOL if r.x.dtype == np.float32 else F64_TOL
    return rel(a, b) <= tol


@pytest.fixture(scope="module")
def server(lib, px):
    cfg = px.ServeConfig(lanes=3, max_batch=64, solo_elements=SOLO, inflight_bytes=256 << 20)
    assert lib.parallax_serve_start(C.byref(cfg)) == px.OK
    yield lib
    assert lib.parallax_serve_stop() == px.OK


def run_alone(lib, px, reqs):
    for r in reqs:
        assert lib.parallax_serve_call(C.byref(r.req)) == px.OK, r.spec


def run_mixed(lib, px, reqs, threads=8):
    errors = []

    def worker(chunk):
        tickets = []
        for r in chunk:
            t = C.c_uint64()
            st = lib.parallax_serve_submit(C.byref(r.req), C.byref(t))
            if st != px.OK:
                errors.append((r.spec, st))
                continue
            tickets.append((r, t.value))
        for r, t in tickets:
            st = lib.parallax_serve_wait(t, None)
            if st != px.OK:
                errors.append((r.spec, st))

    ths = [threading.Thread(target=worker, args=(reqs[i::threads],)) for i in range(threads)]
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    assert not errors, errors


def test_alone_equals_mix_equals_oracle(server, px, dev, ox):
    lib = server
    alone = mix(px, dev, ox)
    mixed = mix(px, dev, ox)  # same inputs, fresh buffers (sort and scan work in place)
    run_alone(lib, px, alone)
    s0 = px.ServeStats()
    lib.parallax_serve_get_stats(C.byref(s0))
    run_mixed(lib, px, mixed)
    s1 = px.ServeStats()
    assert lib.parallax_serve_get_stats(C.byref(s1)) == px.OK
    check_outputs(ox, alone, mixed)
    # every request went through a batch (coalesced or alone); whether requests coalesce
    # depends on how many wait when a lane frees up: test_zz_queued_requests_coalesce
    assert s1.batches - s0.batches <= len(mixed)


def check_outputs(ox, alone, mixed):
    """Each request's result is the same alone and in the mix, and matches the oracle."""
    for a, m in zip(alone, mixed):
        ga, gm = a.output(), m.output()
        want = oracle_of(ox, a)
        assert same(a, ga, gm), f"{a.spec} n={a.x.size}: alone and mixed differ"
        if a.kind == "reduce" and a.x.dtype.kind == "f" and a.spec.startswith("reduce:sum"):
            tol = F32_TOL if a.x.dtype == np.float32 else F64_TOL
            assert rel(ga, want) <= tol, a.spec
        elif a.kind in ("scan", "exscan") and a.x.dtype.kind == "f":
            tol = F32_TOL if a.x.dtype == np.float32 else F64_TOL
            assert rel(ga, want) <= tol, a.spec
        else:
            assert same(a, ga, want if a.kind != "reduce" else a.x.dtype.type(want),
                        exact_fp=True), f"{a.spec} n={a.x.size}: differs from the oracle"


def test_admission_by_memory_budget(server, px, dev, ox):
    """Requests that do not fit next to the in-flight ones wait for completions, then run:
    2^24-key sorts (64 MiB of keys + 64 MiB temporary each) against a 256 MiB budget, all
    submitted at once from one thread while the first ones are still sorting."""
    lib = server
    n = 1 << 24
    reqs = [Req(px, dev, "sort:u32", make(ox, "u32", n, 900 + i), "sort") for i in range(5)]
    s0 = px.ServeStats()
    lib.parallax_serve_get_stats(C.byref(s0))
    tickets = []
    for r in reqs:
        t = C.c_uint64()
        assert lib.parallax_serve_submit(C.byref(r.req), C.byref(t)) == px.OK
        tickets.append(t.value)
    for t in tickets:
        assert lib.parallax_serve_wait(t, None) == px.OK
    s1 = px.ServeStats()
    lib.parallax_serve_get_stats(C.byref(s1))
    assert s1.memory_waits > s0.memory_waits
    assert s1.peak_inflight_bytes <= 256 << 20
    for r in reqs[:2]:
        assert np.array_equal(r.output(), ox.sort(r.x))


def test_served_equals_plain_abi(server, px, dev, ox):
    lib = server
    x = make(ox, "i64", 50000, 77)
    r = Req(px, dev, "reduce:sum:i64", x, "reduce")
    assert lib.parallax_serve_call(C.byref(r.req)) == px.OK
    out = (C.c_ubyte * 8)()
    d = dev.put(x)
    lib.parallax_reduce(px.builtin("reduce:sum:i64"), d.data_ptr(), x.size, 8, out)
    px.check()
    assert r.output() == np.frombuffer(bytes(out), np.int64)[0] == ox.reduce_sum(x)


def test_poll_until_finished(server, px, dev, ox):
    """parallax_serve_poll: not finished (ticket kept) until the request completes, then the
    status and result parallax_serve_wait would give; an empty request is finished at once."""
    lib = server
    x = make(ox, "f64", 300001, 78)
    r = Req(px, dev, "reduce:sum:f64", x, "reduce")
    t = C.c_uint64()
    assert lib.parallax_serve_submit(C.byref(r.req), C.byref(t)) == px.OK
    fin, done, polls = C.c_int(0), C.c_uint64(0), 0
    while True:
        st = lib.parallax_serve_poll(t.value, C.byref(fin), C.byref(done))
        polls += 1
        if fin.value:
            break
        assert st == px.OK
    assert st == px.OK and done.value > 0 and polls >= 1
    assert np.isclose(r.output(), ox.reduce_sum(x), rtol=1e-12)
    e = Req(px, dev, "reduce:sum:f64", x[:0], "reduce")
    assert lib.parallax_serve_submit(C.byref(e.req), C.byref(t)) == px.OK
    assert lib.parallax_serve_poll(t.value, C.byref(fin), None) == px.OK and fin.value == 1
    assert lib.parallax_serve_poll(0, C.byref(fin), None) == px.ERR_INVALID_ARGUMENT
    lib.parallax_clear_error()


def test_errors(server, px, dev):
    lib = server
    r = px.Request()
    r.kernel = None
    assert lib.parallax_serve_call(C.byref(r)) == px.ERR_INVALID_HANDLE
    host = np.arange(100, dtype=np.float32)
    r.kernel = px.builtin("reduce:sum:f32")
    r.input = host.ctypes.data
    r.count = 100
    assert lib.parallax_serve_call(C.byref(r)) == px.ERR_INVALID_ARGUMENT
    lib.parallax_clear_error()


def test_zz_stop_then_submit_is_refused(lib, px, dev):
    """Runs after the module's server stopped (collected last in this file)."""
    cfg = px.ServeConfig()
    assert lib.parallax_serve_start(C.byref(cfg)) == px.OK
    assert lib.parallax_serve_stop() == px.OK
    d = dev.put(np.ones(10, np.float32))
    r = px.Request()
    r.kernel = px.builtin("reduce:sum:f32")
    r.input = d.data_ptr()
    r.count = 10
    t = C.c_uint64()
    assert lib.parallax_serve_submit(C.byref(r), C.byref(t)) == px.ERR_SHUTDOWN
    lib.parallax_clear_error()


def test_zz_wait_after_stop_returns_the_status(lib, px, ox, dev):
    """A request submitted before parallax_serve_stop() is finished by stop; waiting on its
    ticket afterwards returns its status and result (and frees it) instead of failing."""
    cfg = px.ServeConfig()
    assert lib.parallax_serve_start(C.byref(cfg)) == px.OK
    x = make(ox, "i32", 70001, 91)
    d = dev.put(x)
    dev.torch.cuda.synchronize()
    out = (C.c_ubyte * 8)()
    r = px.Request()
    r.kernel = px.builtin("reduce:sum:i32")
    r.input = d.data_ptr()
    r.count = x.size
    r.result = C.cast(out, C.c_void_p)
    t = C.c_uint64()
    assert lib.parallax_serve_submit(C.byref(r), C.byref(t)) == px.OK
    assert lib.parallax_serve_stop() == px.OK
    done = C.c_uint64()
    assert lib.parallax_serve_wait(t.value, C.byref(done)) == px.OK
    assert done.value > 0
    assert np.frombuffer(bytes(out), np.int32, 1)[0] == ox.reduce_sum(x)


def test_zz_queued_requests_coalesce(lib, px, dev, ox):
    """Requests that queue while the only lane is busy (behind a 2^26-key sort) are taken
    as coalesced segmented launches, and every result is still the one it has alone."""
    lib.parallax_serve_stop()
    cfg = px.ServeConfig(lanes=1, max_batch=64, solo_elements=SOLO, inflight_bytes=4 << 30,
                         schedulers=1)
    assert lib.parallax_serve_start(C.byref(cfg)) == px.OK
    try:
        alone = mix(px, dev, ox, seed0=700)
        queued = mix(px, dev, ox, seed0=700)
        run_alone(lib, px, alone)
        big = dev.put(ox.gen("i64_full", 77, 1 << 26))
        dev.torch.cuda.synchronize()
        r = px.Request()
        r.kernel = px.builtin("sort:i64")
        r.input = big.data_ptr()
        r.count = 1 << 26
        s0 = px.ServeStats()
        lib.parallax_serve_get_stats(C.byref(s0))
        t_big = C.c_uint64()
        assert lib.parallax_serve_submit(C.byref(r), C.byref(t_big)) == px.OK
        run_mixed(lib, px, queued, threads=1)
        assert lib.parallax_serve_wait(t_big.value, None) == px.OK
        s1 = px.ServeStats()
        assert lib.parallax_serve_get_stats(C.byref(s1)) == px.OK
        check_outputs(ox, alone, queued)
        assert s1.coalesced_requests > s0.coalesced_requests
        assert s1.batches - s0.batches < len(queued) + 1
    finally:
        assert lib.parallax_serve_stop() == px.OK

