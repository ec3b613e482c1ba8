"""Parity of the sm_100a primitives with the CPU oracle, through the C ABI, on device
pointers. Integer / ordering results bit-exact; fp32 sums and prefixes within 1e-5 and fp64
within 1e-12 max relative error of the compensated fp64 oracle."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import cases
from cases import F32_TOL, F64_TOL

pytestmark = pytest.mark.gpu

EDGE_SIZES = [1, 2, 3, 5, 31, 255, 256, 1000, 1535, 1536, 1537, 3071, 3072, 3073, 4095, 4096,
              4097, 12289, 65543, 1 << 20, (1 << 20) + 12345]
DTYPES = {"f32": np.float32, "f64": np.float64, "i32": np.int32, "i64": np.int64,
          "u32": np.uint32, "u64": np.uint64}


def make(ox, t: str, n: int, seed: int = 1) -> np.ndarray:
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


def reduce_dev(lib, px, h, d, n, dtype):
    out = (C.c_ubyte * 8)()
    lib.parallax_reduce(h, d.data_ptr(), n, np.dtype(dtype).itemsize, out)
    px.check("parallax_reduce")
    return np.frombuffer(bytes(out), dtype=dtype, count=1)[0]


@pytest.mark.parametrize("t", list(DTYPES))
@pytest.mark.parametrize("n", EDGE_SIZES)
def test_reduce_sum(lib, px, ox, dev, t, n):
    x = make(ox, t, n)
    got = reduce_dev(lib, px, px.builtin(f"reduce:sum:{t}"), dev.put(x), n, x.dtype)
    want = ox.reduce_sum(x)
    if t == "f32":
        assert abs(float(got) - want) <= F32_TOL * abs(want)
    elif t == "f64":
        assert abs(float(got) - want) <= F64_TOL * abs(want)
    else:
        assert got == want


@pytest.mark.parametrize("t", list(DTYPES))
@pytest.mark.parametrize("op", ["max", "min"])
@pytest.mark.parametrize("n", [1, 7, 3073, 1 << 20])
def test_reduce_max_min(lib, px, ox, dev, t, op, n):
    x = make(ox, t, n, seed=2)
    got = reduce_dev(lib, px, px.builtin(f"reduce:{op}:{t}"), dev.put(x), n, x.dtype)
    assert got == ox.reduce_minmax(x, op == "max")


@pytest.mark.parametrize("offset", [1, 2, 3])
def test_reduce_unaligned_pointer(lib, px, ox, dev, offset):
    x = make(ox, "i32", 100000)
    d = dev.put(np.concatenate([np.zeros(offset, np.int32), x]))
    out = (C.c_ubyte * 8)()
    lib.parallax_reduce(px.builtin("reduce:sum:i32"), d.data_ptr() + 4 * offset, x.size, 4, out)
    px.check()
    assert np.frombuffer(bytes(out), np.int32, 1)[0] == ox.reduce_sum(x)


def test_reduce_is_deterministic(lib, px, ox, dev):
    x = make(ox, "f32", (1 << 22) + 3)
    d = dev.put(x)
    h = px.builtin("reduce:sum:f32")
    vals = {reduce_dev(lib, px, h, d, x.size, np.float32).tobytes() for _ in range(5)}
    assert len(vals) == 1


def scan_dev(lib, px, dev, t, x, exclusive, init=0):
    n = x.size
    d = dev.put(x)
    h = px.builtin(f"scan:{t}")
    if exclusive:
        o = dev.empty(x.nbytes)
        iv = np.array([init], dtype=x.dtype)
        lib.parallax_exclusive_scan(h, h, h, d.data_ptr(), o.data_ptr(), n, x.itemsize,
                                    iv.ctypes.data)
        px.check("parallax_exclusive_scan")
        return dev.get(o, x.dtype, n)
    lib.parallax_scan(h, h, d.data_ptr(), n, x.itemsize)
    px.check("parallax_scan")
    return dev.get(d, x.dtype, n)


@pytest.mark.parametrize("t", list(DTYPES))
@pytest.mark.parametrize("n", EDGE_SIZES)
@pytest.mark.parametrize("exclusive", [False, True])
def test_scan(lib, px, ox, dev, t, n, exclusive):
    x = make(ox, t, n, seed=3)
    init = 5 if exclusive else 0
    got = scan_dev(lib, px, dev, t, x, exclusive, init)
    want = ox.scan(x, exclusive=exclusive, init=init)
    if t in ("f32", "f64"):
        tol = F32_TOL if t == "f32" else F64_TOL
        assert ox.max_rel_err(got, want) <= tol
    else:
        assert np.array_equal(got, want)


@pytest.mark.parametrize("n", [1000, 100003])
def test_scan_unaligned_falls_back_to_plain_loads(lib, px, ox, dev, n):
    x = make(ox, "i32", n, seed=4)
    d = dev.put(np.concatenate([np.zeros(1, np.int32), x]))
    h = px.builtin("scan:i32")
    lib.parallax_scan(h, h, d.data_ptr() + 4, n, 4)
    px.check()
    assert np.array_equal(dev.get(d, np.int32, n + 1)[1:], ox.scan(x))


def compact_dev(lib, px, dev, spec, x):
    n = x.size
    d = dev.put(x)
    o = dev.empty(x.nbytes)
    h = px.builtin(spec)
    k = lib.parallax_copy_if(h, h, h, h, d.data_ptr(), o.data_ptr(), n, x.itemsize,
                             int(x.dtype.kind == "f"))
    px.check("parallax_copy_if")
    return dev.get(o, x.dtype, n), int(k)


PREDS = [  # (spec tail, oracle kind, c, m, r)
    ("gt:0.5", "P_GT", 0.5, 1, 0),
    ("lt:0", "P_LT", 0.0, 1, 0),
    ("mod:3:0", "P_MOD", 0.0, 3, 0),
    ("nonzero", "P_NONZERO", 0.0, 1, 0),
]


@pytest.mark.parametrize("t", ["i32", "u32", "i64"])
@pytest.mark.parametrize("m", [1, 2, 3, 5, 7, 10, 641, 65537, 6700417, 2**31 - 1, -1, -3, -7,
                               -(2**31) + 1, 2**31, 2**32 - 1, -(2**32) + 5])
def test_modulo_predicate_divisors(lib, px, ox, dev, t, m):
    """x % m == r through the multiply-high remainder and, for r == 0, the multiply-by-inverse
    divisibility test (compaction and the count pass of partition): every divisor class,
    both signs, the extreme values of the type, exact multiples of m."""
    x = make(ox, t, 100003, seed=23)
    info = np.iinfo(x.dtype)
    x[:6] = np.array([0, 1, info.max, info.min, info.max - 1, info.min + 1]).astype(x.dtype)
    if t == "i32":
        x[6:8] = np.array([-1, -2], dtype=np.int32)
    # exact multiples of m (both signs where the type has them) and their neighbours, so the
    # zero-remainder test sees true cases for every divisor
    k = np.arange(-40, 41, dtype=np.int64)
    mult = (k * m).astype(np.int64)
    mult = mult[(mult >= int(info.min)) & (mult <= int(info.max))]
    near = np.concatenate([mult, mult[mult < int(info.max)] + 1, mult[mult > int(info.min)] - 1])
    x[8:8 + near.size] = near.astype(x.dtype)
    for r in (0, 1, 2, -1):
        spec = f"copy_if:{t}:mod:{m}:{r}"
        got, k = compact_dev(lib, px, dev, spec, x)
        want, wk = ox.compact(x, ox.COPY_IF, ox.P_MOD, 0.0, m, r)
        assert k == wk, (spec, k, wk)
        assert np.array_equal(got[:k], want[:k]), spec
        # partition counts with the count_if kernel first, then scatters both sides
        got, k = compact_dev(lib, px, dev, f"partition:{t}:mod:{m}:{r}", x)
        want, wk = ox.compact(x, ox.PARTITION, ox.P_MOD, 0.0, m, r)
        assert k == wk and np.array_equal(got, want), f"partition {spec}"


@pytest.mark.parametrize("t", list(DTYPES))
@pytest.mark.parametrize("n", [1, 2, 33, 3072, 3073, 4097, 65543, (1 << 20) + 7])
@pytest.mark.parametrize("mode", ["copy_if", "remove_if", "partition"])
@pytest.mark.parametrize("pred", PREDS, ids=[p[0] for p in PREDS])
def test_compaction(lib, px, ox, dev, t, n, mode, pred):
    tail, kind, c, m, r = pred
    if tail.startswith("mod") and t in ("f32", "f64"):
        pytest.skip("modulo predicate is integer-only")
    x = make(ox, t, n, seed=5)
    if t == "i32":
        x = x // 3  # some zeros for `nonzero`
    got, k = compact_dev(lib, px, dev, f"{mode}:{t}:{tail}", x)
    omode = {"copy_if": ox.COPY_IF, "remove_if": ox.REMOVE_IF, "partition": ox.PARTITION}[mode]
    want, wk = ox.compact(x, omode, getattr(ox, kind), c, m, r)
    assert k == wk
    written = n if mode == "partition" else k
    assert np.array_equal(got[:written], want[:written])


@pytest.mark.parametrize("t", list(DTYPES))
@pytest.mark.parametrize("n", [1, 2, 3, 1000, 3072, 3073, 65543, (1 << 20) + 5])
def test_unique(lib, px, ox, dev, t, n):
    x = np.sort(make(ox, t, n, seed=6))
    if t in ("i32", "i64", "u32", "u64"):
        x = np.sort(x // x.dtype.type(7) if t != "i64" else x >> 40)
    else:
        x = np.sort(np.round(x * 50) / 50).astype(x.dtype)
    got, k = compact_dev(lib, px, dev, f"unique:{t}", x)
    want, wk = ox.compact(x, ox.UNIQUE)
    assert k == wk and np.array_equal(got[:k], want[:k])


def test_copy_if_empty_and_all(lib, px, ox, dev):
    x = np.arange(10000, dtype=np.int32)
    got, k = compact_dev(lib, px, dev, "copy_if:i32:lt:0", x)
    assert k == 0
    got, k = compact_dev(lib, px, dev, "copy_if:i32:ge:0", x)
    assert k == x.size and np.array_equal(got, x)


def sort_dev(lib, px, dev, spec, x):
    d = dev.put(x)
    lib.parallax_sort(px.builtin(spec), d.data_ptr(), x.size, x.itemsize)
    px.check("parallax_sort")
    return dev.get(d, x.dtype, x.size)


@pytest.mark.parametrize("t", list(DTYPES))
@pytest.mark.parametrize("n", [2, 3, 17, 4095, 4096, 4097, 8192, 12289, 65537, (1 << 20) + 3,
                               1 << 21])
def test_sort(lib, px, ox, dev, t, n):
    x = make(ox, t, n, seed=7)
    if t in ("f32", "f64"):
        x = (x * 2 - 1).astype(x.dtype)
        x[: n // 10] = x[n // 2: n // 2 + n // 10]  # exact duplicates
        if n > 8:
            x[1], x[3] = x.dtype.type(0.0), x.dtype.type(-0.0)
    got = sort_dev(lib, px, dev, f"sort:{t}", x)
    want = ox.sort(x)
    assert np.array_equal(got.view(np.uint8), want.view(np.uint8))


@pytest.mark.parametrize("t,shift", [("u32", 4), ("u32", 8), ("i64", 8)])
@pytest.mark.parametrize("n", [5000, 100003, (1 << 20) + 7])
def test_sort_unaligned_data(lib, px, ox, dev, t, shift, n):
    """Data that is not 16-byte aligned: merge passes alternate between it and the aligned
    temporary (scalar and vector output stores); every layout must give the same order."""
    x = make(ox, t, n, seed=17)
    buf = dev.put(np.concatenate([np.zeros(shift, np.uint8), x.view(np.uint8)]))
    h = px.builtin(f"sort:{t}")
    lib.parallax_sort(h, buf.data_ptr() + shift, n, x.itemsize)
    px.check("unaligned sort")
    got = buf[shift:].cpu().numpy().view(x.dtype)
    assert np.array_equal(got, ox.sort(x))


@pytest.mark.parametrize("n", [2, 1000, 100000, (1 << 20) + 3])
def test_sort_kv_is_stable_by_key(lib, px, ox, dev, n):
    keys = (ox.gen("u32_full", 8, n) % 1000).astype(np.uint64)
    rec = (keys << np.uint64(32)) | np.arange(n, dtype=np.uint64)
    got = sort_dev(lib, px, dev, "sort_kv:u32", rec)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(got & np.uint64(0xFFFFFFFF), order.astype(np.uint64))


@pytest.mark.parametrize("n", [3, 4097, 300001])
def test_sort_kv_keeps_input_order_of_equal_keys_with_random_values(lib, px, ox, dev, n):
    """Stable by key means equal keys keep their input order, not their value order."""
    keys = (ox.gen("u32_full", 9, n) % 50).astype(np.uint64)
    vals = ox.gen("u32_full", 10, n).astype(np.uint64)
    rec = (keys << np.uint64(32)) | vals
    got = sort_dev(lib, px, dev, "sort_kv:u32", rec)
    assert np.array_equal(got, rec[np.argsort(keys, kind="stable")])


@pytest.mark.parametrize("t", list(DTYPES))
@pytest.mark.parametrize("n", [1, 2, 1000, 65543, (1 << 20) + 1])
def test_argminmax(lib, px, ox, dev, t, n):
    x = make(ox, t, n, seed=9)
    if t in ("i32",):
        x = x // 100  # ties
    d = dev.put(x)
    h = px.builtin(f"argminmax:{t}")
    for want_max in (0, 1):
        for want_last in (0, 1):
            got = lib.parallax_argminmax(h, d.data_ptr(), n, x.itemsize, int(x.dtype.kind == "f"),
                                         want_max, want_last)
            px.check()
            assert got == ox.argminmax(x, bool(want_max), bool(want_last))


@pytest.mark.parametrize("t", ["f32", "i32", "i64", "u64"])
@pytest.mark.parametrize("n", [1, 1000, 65543, (1 << 20) + 9])
def test_find_and_count(lib, px, ox, dev, t, n):
    x = make(ox, t, n, seed=10)
    d = dev.put(x)
    c = 0.999 if t == "f32" else (990 if t == "i32" else 0)
    kind = "gt"
    h = px.builtin(f"find:{t}:{kind}:{c}")
    for negate in (0, 1):
        got = lib.parallax_find(h, d.data_ptr(), n, x.itemsize, negate, None)
        px.check()
        assert got == ox.find(x, ox.P_GT, c, negate=bool(negate))
    v = np.array([x[n // 2]], dtype=x.dtype)
    got = lib.parallax_find(h, d.data_ptr(), n, x.itemsize, 0, v.ctypes.data)
    px.check()
    assert got == ox.find(x, ox.P_EQ, float(v[0]) if t == "f32" else int(v[0]))


@pytest.mark.parametrize("t", ["f32", "f64", "i32", "u64"])
@pytest.mark.parametrize("n", [1, 4, 1000, (1 << 20) + 3])
def test_mismatch(lib, px, ox, dev, t, n):
    a = make(ox, t, n, seed=11)
    b = a.copy()
    h = px.builtin(f"mismatch:{t}")
    da = dev.put(a)
    for pos in [None, n - 1, n // 2, 0]:
        bb = b.copy()
        if pos is not None:
            bb[pos] = bb[pos] + bb.dtype.type(1)
        db = dev.put(bb)  # keep the tensor alive while its pointer is in use
        got = lib.parallax_mismatch(h, da.data_ptr(), db.data_ptr(), n, a.itemsize)
        px.check()
        assert got == ox.mismatch(a, bb)
