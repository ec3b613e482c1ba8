"""CPU oracle (test infrastructure only).

Loads oracle/liboracle.so (the CPU restatement in oracle.cpp) and, when present,
oracle/_ref/libparallax_ref.so (the reference's own stdpar.hpp host fallbacks, built by
oracle/Makefile from the reference tree) and oracle/libpstl_baseline.so (the primitives
under std::execution::par, a timed baseline). Only tests, __graft_entry__.smoke() and
bench.py's CPU-baseline leg use this module, and only as the checker or the timed CPU
baseline; the runtime never calls it.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libparallax_ref.so"

# predicate kinds (same numbering as the runtime)
P_GT, P_GE, P_LT, P_LE, P_EQ, P_NE, P_MOD, P_NONZERO = 1, 2, 3, 4, 5, 6, 7, 8
# compaction modes
COPY_IF, REMOVE_IF, PARTITION, UNIQUE = 0, 1, 2, 3

SUFFIX = {np.float32: "f32", np.float64: "f64", np.int32: "i32", np.int64: "i64",
          np.uint32: "u32", np.uint64: "u64"}

_ox = None
_ref = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def ox() -> C.CDLL:
    global _ox
    if _ox is None:
        if not ORACLE_SO.exists():
            build()
        _ox = C.CDLL(str(ORACLE_SO))
    return _ox


PSTL_SO = HERE / "libpstl_baseline.so"
_pstl = None


def pstl() -> C.CDLL | None:
    """The primitives under std::execution::par (host C++ library), or None when not built."""
    global _pstl
    if _pstl is None and PSTL_SO.exists():
        _pstl = C.CDLL(str(PSTL_SO))
        _pstl.pstl_backend.restype = C.c_char_p
        _pstl.pstl_threads.restype = C.c_uint
    return _pstl


def ref() -> C.CDLL | None:
    """The reference's compiled host fallbacks, or None when not built here."""
    global _ref
    if _ref is None and REF_SO.exists():
        _ref = C.CDLL(str(REF_SO))
    return _ref


def _p(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def sfx(dtype) -> str:
    return SUFFIX[np.dtype(dtype).type]


# ---- generators ---------------------------------------------------------------------------
def gen(kind: str, seed: int, n: int) -> np.ndarray:
    """Seeded counter-based inputs: f32_unit, f64_unit, i32_pm1000, u32_full, i64_full."""
    dt = {"f32_unit": np.float32, "f64_unit": np.float64, "i32_pm1000": np.int32,
          "u32_full": np.uint32, "i64_full": np.int64}[kind]
    out = np.empty(n, dtype=dt)
    getattr(ox(), "ox_gen_" + kind)(C.c_uint64(seed), C.c_uint64(n), _p(out))
    return out


def gen_u64(seed: int, n: int, start: int = 0) -> np.ndarray:
    out = np.empty(n, dtype=np.uint64)
    ox().ox_gen_u64(C.c_uint64(seed), C.c_uint64(start), C.c_uint64(n), _p(out))
    return out


# ---- primitives ---------------------------------------------------------------------------
def reduce_sum(x: np.ndarray):
    s = sfx(x.dtype)
    if s in ("f32", "f64"):
        f = getattr(ox(), "ox_sum_" + s)
        f.restype = C.c_double
        return f(_p(x), C.c_uint64(x.size))
    w = 32 if s in ("i32", "u32") else 64
    f = getattr(ox(), f"ox_sum_u{w}")
    f.restype = C.c_uint32 if w == 32 else C.c_uint64
    v = f(_p(x), C.c_uint64(x.size))
    return np.array([v], dtype=np.uint32 if w == 32 else np.uint64).view(x.dtype)[0]


def reduce_minmax(x: np.ndarray, want_max: bool):
    s = sfx(x.dtype)
    f = getattr(ox(), "ox_minmax_" + s)
    f.restype = {"f32": C.c_float, "f64": C.c_double, "i32": C.c_int32, "i64": C.c_int64,
                 "u32": C.c_uint32, "u64": C.c_uint64}[s]
    return x.dtype.type(f(_p(x), C.c_uint64(x.size), C.c_int(int(want_max))))


def scan(x: np.ndarray, exclusive: bool = False, init=0) -> np.ndarray:
    """fp types: fp64 compensated prefix (float64 array); integers: wrapped, same dtype."""
    s = sfx(x.dtype)
    n = C.c_uint64(x.size)
    if s in ("f32", "f64"):
        out = np.empty(x.size, dtype=np.float64)
        getattr(ox(), "ox_scan_" + s)(_p(x), _p(out), n, C.c_int(int(exclusive)),
                                      C.c_double(float(init)))
        return out
    w = 32 if s in ("i32", "u32") else 64
    ut = np.uint32 if w == 32 else np.uint64
    out = np.empty(x.size, dtype=ut)
    init_u = np.array([init], dtype=x.dtype).view(ut)[0]
    getattr(ox(), f"ox_scan_u{w}")(_p(x.view(ut)), _p(out), n, C.c_int(int(exclusive)),
                                   (C.c_uint32 if w == 32 else C.c_uint64)(int(init_u)))
    return out.view(x.dtype)


def sort(x: np.ndarray) -> np.ndarray:
    y = np.ascontiguousarray(x).copy()
    getattr(ox(), "ox_sort_" + sfx(x.dtype))(_p(y), C.c_uint64(y.size))
    return y


def _operand(c) -> tuple[C.c_double, C.c_int64]:
    """Predicate operand as (float, exact integer); integers beyond int64 wrap like C."""
    if isinstance(c, (int, np.integer)):
        ci = int(c)
        ci = (ci + (1 << 63)) % (1 << 64) - (1 << 63)
        return C.c_double(float(c)), C.c_int64(ci)
    return C.c_double(float(c)), C.c_int64(int(c))


def compact(x: np.ndarray, mode: int, kind: int = 0, c=0.0, m: int = 1,
            r: int = 0) -> tuple[np.ndarray, int]:
    """Returns (output array of len n, kept count)."""
    out = np.zeros_like(x)
    f = getattr(ox(), "ox_compact_" + sfx(x.dtype))
    f.restype = C.c_uint64
    k = f(_p(x), _p(out), C.c_uint64(x.size), C.c_int(mode), C.c_int(kind), *_operand(c),
          C.c_int64(m), C.c_int64(r))
    return out, int(k)


def count_if(x: np.ndarray, kind: int, c=0.0, m: int = 1, r: int = 0) -> int:
    f = getattr(ox(), "ox_count_" + sfx(x.dtype))
    f.restype = C.c_uint64
    return int(f(_p(x), C.c_uint64(x.size), C.c_int(kind), *_operand(c), C.c_int64(m),
                 C.c_int64(r)))


def find(x: np.ndarray, kind: int, c=0.0, m: int = 1, r: int = 0,
         negate: bool = False) -> int:
    f = getattr(ox(), "ox_find_" + sfx(x.dtype))
    f.restype = C.c_uint64
    return int(f(_p(x), C.c_uint64(x.size), C.c_int(kind), *_operand(c), C.c_int64(m),
                 C.c_int64(r), C.c_int(int(negate))))


def argminmax(x: np.ndarray, want_max: bool, want_last: bool) -> int:
    f = getattr(ox(), "ox_argminmax_" + sfx(x.dtype))
    f.restype = C.c_uint64
    return int(f(_p(x), C.c_uint64(x.size), C.c_int(int(want_max)), C.c_int(int(want_last))))


def mismatch(a: np.ndarray, b: np.ndarray) -> int:
    f = getattr(ox(), "ox_mismatch_" + sfx(a.dtype))
    f.restype = C.c_uint64
    return int(f(_p(a), _p(b), C.c_uint64(a.size)))


def saxpy_gather(records: np.ndarray, a: float, tgt: np.ndarray, host_base: int) -> np.ndarray:
    n = records.size // 4 if records.dtype == np.uint32 else records.nbytes // 16
    y = np.empty(n, dtype=np.float32)
    ox().ox_saxpy_gather(_p(records), C.c_uint64(n), C.c_float(a), _p(tgt),
                         C.c_uint64(host_base), _p(y))
    return y


def max_rel_err(got: np.ndarray, want: np.ndarray, floor: float = 0.0) -> float:
    """max |got - want| / max(|want|, floor) in fp64."""
    g = np.asarray(got, dtype=np.float64)
    w = np.asarray(want, dtype=np.float64)
    den = np.maximum(np.abs(w), floor) if floor else np.abs(w)
    den = np.where(den == 0, 1.0, den)
    return float(np.max(np.abs(g - w) / den)) if g.size else 0.0


# ---- segmented primitives -----------------------------------------------------------------------
# Each applies the per-array oracle above to every segment [offsets[s], offsets[s+1]) of x:
# the per-segment contract is exactly the reference primitive's (stdpar.hpp:146-148 reduce,
# :237-238 exclusive_scan, :319-321 copy_if, :178 sort).
def seg_sum(x: np.ndarray, offsets: np.ndarray) -> np.ndarray:
    """Per-segment sums: float64 (compensated) for fp inputs, wrapped x.dtype for integers;
    empty segments give 0."""
    S = offsets.size - 1
    fp = x.dtype.kind == "f"
    out = np.zeros(S, dtype=np.float64 if fp else x.dtype)
    for s in range(S):
        a, b = int(offsets[s]), int(offsets[s + 1])
        if b > a:
            out[s] = reduce_sum(x[a:b])
    return out


def seg_exscan(x: np.ndarray, offsets: np.ndarray, init=0) -> np.ndarray:
    """Per-segment exclusive scans, each starting at init (float64 for fp inputs)."""
    fp = x.dtype.kind == "f"
    out = np.zeros(x.size, dtype=np.float64 if fp else x.dtype)
    for s in range(offsets.size - 1):
        a, b = int(offsets[s]), int(offsets[s + 1])
        if b > a:
            out[a:b] = scan(x[a:b], exclusive=True, init=init)
    return out


def seg_copy_if(x: np.ndarray, offsets: np.ndarray, kind: int, c=0.0,
                remove: bool = False) -> tuple[list[np.ndarray], np.ndarray]:
    """Kept elements of every segment (in order) and the kept counts."""
    kept, counts = [], np.zeros(offsets.size - 1, dtype=np.uint64)
    for s in range(offsets.size - 1):
        a, b = int(offsets[s]), int(offsets[s + 1])
        out, k = compact(x[a:b], REMOVE_IF if remove else COPY_IF, kind, c)
        kept.append(out[:k])
        counts[s] = k
    return kept, counts


def seg_sort(x: np.ndarray, offsets: np.ndarray) -> np.ndarray:
    y = x.copy()
    for s in range(offsets.size - 1):
        a, b = int(offsets[s]), int(offsets[s + 1])
        if b - a > 1:
            y[a:b] = sort(x[a:b])
    return y
