"""Compiler-emitted kernels through the unchanged C ABI on a B200.

The parallax compiler embeds one kernel image per funnel instantiation and registers it
under the funnel's __PRETTY_FUNCTION__ key at static init (reference
src/kernel/cache.cpp:83-104, include/parallax/runtime.h:96-103). The images here
(tests/images/*.cu, compiled to sm_100a fatbins by tests/images/build_images.py) stand in
for that output. Each test registers an image under the key GCC gives the stdpar funnel
(include/parallax/stdpar.hpp), looks it up, and launches it the way the funnel does:
  launch / launch_with_captures     device_invoke       (stdpar.hpp:46-82)
  launch_transform2(_captures)      device_transform    (stdpar.hpp:88-120)
  copy_if with a registered :flags  device_copy_if / remove_if / partition (stdpar.hpp:300-371;
                                    reference kernel_launcher.cpp:1701-1791)
  :pred transform + ':reduce'       device_count_if     (stdpar.hpp:271-293)
  :xform transform + ':reduce'      device_transform_reduce (stdpar.hpp:241-267)
Transforms whose image also exports its element function as LTO-IR (images/*_lto.cu) run
fused with the reduce that follows them: one launch instead of two.
Results are compared with host computations (bit-exact) and the oracle.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from helpers import Arena

pytestmark = pytest.mark.gpu

IMAGES = Path(__file__).resolve().parent / "images" / "_build"
SZ = "std::size_t = long unsigned int"


def key(sig: str, with_: str, suffix: str = "") -> str:
    return f"{sig} [with {with_}; {SZ}]" + (f":{suffix}" if suffix else "")


INVOKE = "void parallax::detail::device_invoke(T*, std::size_t, F)"
TRANSFORM = "void parallax::detail::device_transform(const Tin*, Tout*, std::size_t, F)"
COPY_IF = "std::size_t parallax::detail::device_copy_if(const T*, T*, std::size_t, Pred)"
REMOVE_IF = "std::size_t parallax::detail::device_remove_if(T*, std::size_t, Pred)"
PARTITION = "std::size_t parallax::detail::device_partition(T*, std::size_t, Pred)"
COUNT_IF = "long int parallax::detail::device_count_if(const T*, std::size_t, Pred)"
TRANSFORM_REDUCE = "U parallax::detail::device_transform_reduce(const T*, std::size_t, F)"

_keep = []  # registered images must outlive the process (the registry borrows them)


def image(name: str):
    p = IMAGES / f"{name}.fatbin"
    if not p.exists():
        pytest.fail(f"{p} not built (python tests/images/build_images.py)")
    data = p.read_bytes()
    data += b"\0" * (-len(data) % 4)
    buf = (C.c_uint32 * (len(data) // 4)).from_buffer_copy(data)
    _keep.append(buf)
    return buf


def register(lib, k: str, name: str):
    buf = image(name)
    lib.parallax_kernel_register(k.encode(), C.cast(buf, C.c_void_p), len(buf))
    h = lib.parallax_kernel_lookup(k.encode())
    assert h, f"lookup of a registered {name} image missed"
    return h


def lookup(lib, k: str):
    return lib.parallax_kernel_lookup(k.encode())


@pytest.fixture
def arena(lib):
    a = Arena(lib)
    yield a
    a.free()


def P(a: np.ndarray) -> int:
    return a.ctypes.data


def rng_f32(n, seed):
    return np.random.default_rng(seed).random(n, dtype=np.float32)


@pytest.mark.parametrize("n", [1, 255, 256, 100003, 1 << 21])
def test_for_each_launch_and_captures(lib, px, arena, n):
    """device_invoke: a captureless functor takes parallax_kernel_launch (variadic), a
    capturing one launch_with_captures with the closure bytes (stdpar.hpp:52-60)."""
    h = register(lib, key(INVOKE, "T = float; F = Affine"), "affine_f32")
    x0 = rng_f32(n, 1)
    data = arena.array(x0)
    lib.parallax_kernel_launch(C.c_void_p(h), C.c_void_p(P(data)), C.c_size_t(n), C.c_size_t(4))
    px.check("parallax_kernel_launch")
    want = x0 * np.float32(2) + np.float32(1)
    assert np.array_equal(data, want)
    cap = np.array([1.5, -0.25], np.float32)  # the functor's bytes {a, b}
    lib.parallax_kernel_launch_with_captures(h, P(data), n, P(cap), cap.nbytes, 4)
    px.check("parallax_kernel_launch_with_captures")
    want = want * np.float32(1.5) + np.float32(-0.25)
    assert np.array_equal(data, want)


def test_kernel_load_returns_a_launchable_handle(lib, px, dev):
    buf = image("affine_f32")
    h = lib.parallax_kernel_load(C.cast(buf, C.c_void_p), len(buf))
    px.check("parallax_kernel_load")
    assert h
    x0 = rng_f32(5000, 2)
    d = dev.put(x0)
    dev.torch.cuda.synchronize()
    lib.parallax_kernel_launch(C.c_void_p(h), C.c_void_p(d.data_ptr()), C.c_size_t(x0.size),
                               C.c_size_t(4))
    px.check()
    assert np.array_equal(dev.get(d, np.float32, x0.size), x0 * np.float32(2) + np.float32(1))


@pytest.mark.parametrize("n", [1, 1000, 65537])
def test_transform2_between_element_sizes(lib, px, arena, dev, n):
    """device_transform: int -> double via launch_transform2 (stdpar.hpp:93-95), on arena
    blocks (coherent: results visible on the host) and on device pointers."""
    h = register(lib, key(TRANSFORM, "Tin = int; Tout = double; F = HalfD"), "half_i32_to_f64")
    x = np.random.default_rng(3).integers(-10**6, 10**6, n, dtype=np.int32)
    want = x.astype(np.float64) * 0.5
    inp, out = arena.array(x), arena.empty(n, np.float64)
    lib.parallax_kernel_launch_transform2(h, P(inp), P(out), n, 4, 8)
    px.check("transform2")
    assert np.array_equal(out, want)
    di, do = dev.put(x), dev.empty(n * 8)
    dev.torch.cuda.synchronize()
    lib.parallax_kernel_launch_transform2(h, di.data_ptr(), do.data_ptr(), n, 4, 8)
    px.check("transform2 device")
    assert np.array_equal(dev.get(do, np.float64, n), want)


def test_transform_variadic_same_element_size(lib, px, arena):
    h = register(lib, key(TRANSFORM, "Tin = float; Tout = float; F = Affine"), "affine_f32")
    x0 = rng_f32(4097, 4)
    inp, out = arena.array(x0), arena.empty(x0.size, np.float32)
    lib.parallax_kernel_launch_transform(C.c_void_p(h), C.c_void_p(P(inp)), C.c_void_p(P(out)),
                                         C.c_size_t(x0.size), C.c_size_t(4))
    px.check("parallax_kernel_launch_transform")
    assert np.array_equal(out, x0 * np.float32(2) + np.float32(1))
    assert np.array_equal(inp, x0)


@pytest.mark.parametrize("n", [1, 4096, 1 << 20])
def test_transform2_captures_relocates_stored_host_pointers(lib, px, ox, arena, n):
    """Records {float x; u32 pad; float* p} whose p are HOST addresses of another arena
    block: the image relocates them in the kernel (dev_base + (p - host_base), reference
    kernel_launcher.cpp:15-32) and reads the gathered value; y = a*x + *p bit-exact."""
    h = register(lib, key(TRANSFORM, "Tin = Rec; Tout = float; F = Saxpy"), "saxpy_gather_f32")
    rng = np.random.default_rng(5)
    tgt = arena.array(rng.random(n, dtype=np.float32))
    rec = np.zeros(n * 4, np.uint32)
    rec[0::4] = rng.random(n, dtype=np.float32).view(np.uint32)
    ptrs = P(tgt) + 4 * rng.integers(0, n, n).astype(np.uint64)
    rec.view(np.uint64)[1::2] = ptrs
    recs = arena.array(rec)
    out = arena.empty(n, np.float32)
    a = np.array([1.5], np.float32)
    lib.parallax_kernel_launch_transform2_captures(h, P(recs), P(out), n, 16, 4, P(a), 4)
    px.check("transform2_captures")
    want = ox.saxpy_gather(rec, 1.5, np.array(tgt), P(tgt))
    assert np.array_equal(out, want)


def test_writes_through_stored_pointers_reach_the_host(lib, px, arena):
    """An image that writes another arena block through stored pointers: the call downloads
    every coherent block afterwards (the reference's whole-arena invalidate,
    src/memory/arena.cpp:296-304), so the host sees the writes."""
    h = register(lib, key(INVOKE, "T = float*; F = Bump"), "bump_through_ptr_f32")
    m = 100000
    tgt = arena.array(np.zeros(m, np.float32))
    idx = np.random.default_rng(6).permutation(m)[: m // 2]  # one writer per element
    ptrs = arena.array((P(tgt) + 4 * idx.astype(np.uint64)).astype(np.uint64))
    lib.parallax_kernel_launch(C.c_void_p(h), C.c_void_p(P(ptrs)), C.c_size_t(idx.size),
                               C.c_size_t(8))
    px.check("launch through pointers")
    want = np.zeros(m, np.float32)
    want[idx] = 1.0
    assert np.array_equal(tgt, want)


def funnel_handles(lib, sig: str, with_: str, image_name: str):
    """The four handles a compaction funnel looks up (stdpar.hpp:302-305): `:flags` is the
    registered image, the other three resolve to built-in generic kernels."""
    kf = register(lib, key(sig, with_, "flags"), image_name)
    ks, ka, kc = (lookup(lib, key(sig, with_, s)) for s in ("scan", "add", "scatter"))
    assert ks and ka and kc
    return kf, ks, ka, kc


SIZES = [1, 2, 3, 1000, 28671, 28672, 28673, 65543, (1 << 20) + 7]


def i32_input(n, seed):
    return np.random.default_rng(seed).integers(-1000, 1001, n, dtype=np.int32)


@pytest.mark.parametrize("n", SIZES)
def test_copy_if_remove_if_partition_with_registered_flags(lib, px, ox, arena, n):
    x = i32_input(n, 7)
    # copy_if(x % 3 == 0)
    hs = funnel_handles(lib, COPY_IF, "T = int; Pred = Mod3", "flags_mod3_i32")
    inp, out = arena.array(x), arena.array(np.full(n, -7, np.int32))
    k = lib.parallax_copy_if(*hs, P(inp), P(out), n, 4, 0)
    px.check("copy_if")
    want, wk = ox.compact(x, ox.COPY_IF, ox.P_MOD, 0.0, 3, 0)
    assert k == wk and np.array_equal(out[:k], want[:k])
    assert np.all(out[k:] == -7)
    # remove_if(x % 3 == 0): the compiler's flags kernel flags the elements to keep
    hs = funnel_handles(lib, REMOVE_IF, "T = int; Pred = Mod3", "flags_not_mod3_i32")
    out[:] = -7
    k = lib.parallax_copy_if(*hs, P(inp), P(out), n, 4, 0)
    px.check("remove_if")
    want, wk = ox.compact(x, ox.REMOVE_IF, ox.P_MOD, 0.0, 3, 0)
    assert k == wk and np.array_equal(out[:k], want[:k])
    # partition(x < 0): stable, every element written, returns the kept count
    hs = funnel_handles(lib, PARTITION, "T = int; Pred = Neg", "flags_neg_i32")
    k = lib.parallax_copy_if(*hs, P(inp), P(out), n, 4, 0)
    px.check("partition")
    want, wk = ox.compact(x, ox.PARTITION, ox.P_LT, 0.0)
    assert k == wk and np.array_equal(out, want)


@pytest.mark.parametrize("n", [1, 5, 14335, 14336, 14337, 100003])
def test_registered_flags_on_8_byte_elements(lib, px, dev, n):
    x = np.random.default_rng(8).integers(-(1 << 62), 1 << 62, n, dtype=np.int64)
    keep = (x & 1) != 0
    d, o = dev.put(x), dev.empty(x.nbytes)
    dev.torch.cuda.synchronize()
    hs = funnel_handles(lib, COPY_IF, "T = long int; Pred = Odd", "flags_odd_i64")
    k = lib.parallax_copy_if(*hs, d.data_ptr(), o.data_ptr(), n, 8, 0)
    px.check("copy_if i64")
    assert k == keep.sum() and np.array_equal(dev.get(o, np.int64, k), x[keep])
    hs = funnel_handles(lib, PARTITION, "T = long int; Pred = Odd", "flags_odd_i64")
    k = lib.parallax_copy_if(*hs, d.data_ptr(), o.data_ptr(), n, 8, 0)
    px.check("partition i64")
    assert k == keep.sum()
    assert np.array_equal(dev.get(o, np.int64, n), np.concatenate([x[keep], x[~keep]]))


def test_reference_flags_shader_predicate(lib, px, ox, arena):
    """The reference's own flags shader keeps x > 0.5 (shaders/flags.comp:14-18)."""
    x = rng_f32((1 << 20) + 3, 9)
    hs = funnel_handles(lib, COPY_IF, "T = float; Pred = GtHalf", "flags_gt_half_f32")
    inp, out = arena.array(x), arena.empty(x.size, np.float32)
    k = lib.parallax_copy_if(*hs, P(inp), P(out), x.size, 4, 1)
    px.check()
    want, wk = ox.compact(x, ox.COPY_IF, ox.P_GT, 0.5)
    assert k == wk and np.array_equal(out[:k], want[:k])


def test_count_if_funnel(lib, px, arena):
    """device_count_if: the registered :pred transform writes 1/0 ints and ':reduce' resolves
    to the built-in int '+' reduce (stdpar.hpp:271-293)."""
    sig_with = "T = float; Pred = GtHalf"
    kp = register(lib, key(COUNT_IF, sig_with, "pred"), "pred_gt_half_f32")
    kr = lookup(lib, key(COUNT_IF, sig_with, "reduce"))
    assert kr
    x = rng_f32(777777, 10)
    inp, flags = arena.array(x), arena.empty(x.size, np.int32)
    lib.parallax_kernel_launch_transform2(kp, P(inp), P(flags), x.size, 4, 4)
    px.check("count_if pred")
    res = np.zeros(1, np.int32)
    lib.parallax_reduce(kr, P(flags), x.size, 4, P(res))
    px.check("count_if reduce")
    assert res[0] == np.count_nonzero(x > np.float32(0.5))


def test_registered_flags_refuse_other_element_sizes(lib, px, dev):
    """Registered flags drive a compaction of 4- or 8-byte words; other element sizes are an
    error the caller can see, never a silent zero-length result."""
    kf = register(lib, key(COPY_IF, "T = short int; Pred = Pos", "flags"), "flags_neg_i32")
    _, ks, ka, kc = funnel_handles(lib, COPY_IF, "T = int; Pred = Neg", "flags_neg_i32")
    hs = (kf, ks, ka, kc)
    d = dev.put(np.zeros(64, np.int16))
    o = dev.empty(128)
    dev.torch.cuda.synchronize()
    assert lib.parallax_copy_if(*hs, d.data_ptr(), o.data_ptr(), 64, 2, 0) == 0
    assert lib.parallax_last_error() == px.ERR_UNSUPPORTED
    lib.parallax_clear_error()


# ---- fused transform + reduce (images that export parallax_elem as LTO-IR) ---------------------

def funnel_call(lib, px, kx, kr, inp, out, n, in_es, out_es, res):
    """The funnel's two calls (stdpar.hpp:251-259); returns the kernels they launched."""
    before = lib.parallax_launch_count()
    lib.parallax_kernel_launch_transform2(kx, P(inp), P(out), n, in_es, out_es)
    px.check("funnel transform")
    lib.parallax_reduce(kr, P(out), n, out_es, P(res))
    px.check("funnel reduce")
    return lib.parallax_launch_count() - before


@pytest.mark.parametrize("n", [1, 255, 2049, 1_000_003])
def test_transform_reduce_funnel_runs_as_one_fused_pass(lib, px, arena, n):
    sig_with = "T = int; U = double; F = HalfL"
    kx = register(lib, key(TRANSFORM_REDUCE, sig_with, "xform"), "xform_half_i32_to_f64_lto")
    kr = lookup(lib, key(TRANSFORM_REDUCE, sig_with, "reduce"))
    assert kr
    x = np.random.default_rng(31).integers(-2**31, 2**31, n, dtype=np.int64).astype(np.int32)
    inp, out = arena.array(x), arena.empty(n, np.float64)
    res = np.zeros(1, np.float64)
    assert funnel_call(lib, px, kx, kr, inp, out, n, 4, 8, res) == 1
    # multiples of 0.5 below 2^52: the fp64 sum is exact in any order
    assert res[0] == float(x.astype(np.int64).sum()) * 0.5


@pytest.mark.parametrize("n", [1, 4097, 777_777])
def test_count_if_funnel_runs_as_one_fused_pass(lib, px, arena, n):
    sig_with = "T = float; Pred = GtHalfL"
    kp = register(lib, key(COUNT_IF, sig_with, "pred"), "pred_gt_half_f32_lto")
    kr = lookup(lib, key(COUNT_IF, sig_with, "reduce"))
    x = rng_f32(n, 12)
    inp, flags = arena.array(x), arena.empty(n, np.int32)
    res = np.zeros(1, np.int32)
    assert funnel_call(lib, px, kp, kr, inp, flags, n, 4, 4, res) == 1
    assert res[0] == np.count_nonzero(x > np.float32(0.5))


def test_fused_integer_sum_equals_two_pass_sum(lib, px, arena, dev):
    """x * x over int64 (wrapping), summed with wrap-around: the fused pass and the two-pass
    path (the same image under a transform key that is not fused, then the built-in reduce)
    give the same bits, and both equal the host's modular sum."""
    n = 3_000_001
    x = np.random.default_rng(32).integers(-2**62, 2**62, n, dtype=np.int64)
    sig_with = "T = long int; U = long int; F = SqL"
    kx = register(lib, key(TRANSFORM_REDUCE, sig_with, "xform"), "xform_sq_i64_lto")
    kr = lookup(lib, key(TRANSFORM_REDUCE, sig_with, "reduce"))
    inp, out = arena.array(x), arena.empty(n, np.int64)
    fused = np.zeros(1, np.int64)
    assert funnel_call(lib, px, kx, kr, inp, out, n, 8, 8, fused) == 1
    kt = register(lib, key(TRANSFORM, "Tin = long int; Tout = long int; F = SqL"), "xform_sq_i64_lto")
    two = np.zeros(1, np.int64)
    assert funnel_call(lib, px, kt, px.builtin("reduce:sum:i64"), inp, out, n, 8, 8, two) == 2
    xu = x.view(np.uint64)
    with np.errstate(over="ignore"):
        want = np.array([(xu * xu).sum(dtype=np.uint64)], np.uint64).view(np.int64)[0]
    assert fused[0] == two[0] == want
    assert np.array_equal(out.view(np.uint64), xu * xu)  # the two-pass transform's output


def test_held_back_transform_runs_before_any_other_call(lib, px, arena):
    """A funnel transform is held back only until the next call on the thread: a different
    call (here a max reduce of its output, then a free of its input) sees the transform's
    output exactly as if it had run at once."""
    sig_with = "T = int; U = double; F = HalfM"
    kx = register(lib, key(TRANSFORM_REDUCE, sig_with, "xform"), "xform_half_i32_to_f64_lto")
    x = np.random.default_rng(33).integers(-10**6, 10**6, 100_003, dtype=np.int64).astype(np.int32)
    inp, out = arena.array(x), arena.empty(x.size, np.float64)
    lib.parallax_kernel_launch_transform2(kx, P(inp), P(out), x.size, 4, 8)
    px.check("held-back transform")
    res = np.zeros(1, np.float64)
    lib.parallax_reduce(px.builtin("reduce:max:f64"), P(out), x.size, 8, P(res))
    px.check("max of the transform's output")
    assert res[0] == x.max() * 0.5
    assert np.array_equal(out, x.astype(np.float64) * 0.5)
    # held back again, then the input block is freed: the transform runs before the free
    out[:] = 0
    lib.parallax_kernel_launch_transform2(kx, P(inp), P(out), x.size, 4, 8)
    lib.parallax_arena_free(C.c_void_p(P(inp)))
    arena.blocks.remove(P(inp))
    px.check("free after a held-back transform")
    assert np.array_equal(out, x.astype(np.float64) * 0.5)


def test_transform_without_element_function_runs_two_passes(lib, px, arena):
    """The same funnel with an image that exports no parallax_elem (plain sm_100a) runs its
    transform and its reduce as two launches and gives the same sum."""
    sig_with = "T = int; U = double; F = HalfP"
    kx = register(lib, key(TRANSFORM_REDUCE, sig_with, "xform"), "half_i32_to_f64")
    kr = lookup(lib, key(TRANSFORM_REDUCE, sig_with, "reduce"))
    x = np.random.default_rng(34).integers(-2**31, 2**31, 500_001, dtype=np.int64).astype(np.int32)
    inp, out = arena.array(x), arena.empty(x.size, np.float64)
    res = np.zeros(1, np.float64)
    assert funnel_call(lib, px, kx, kr, inp, out, x.size, 4, 8, res) == 2
    assert res[0] == float(x.astype(np.int64).sum()) * 0.5
    assert np.array_equal(out, x.astype(np.float64) * 0.5)
