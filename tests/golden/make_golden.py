"""Generates tests/golden/ref_vectors.npz from the reference's own CPU path.

Runs the reference's stdpar.hpp host fallbacks (compiled by oracle/Makefile into
oracle/_ref/libparallax_ref.so from the read-only reference tree) on seeded inputs and
stores inputs' generator parameters plus the reference's outputs. The committed file pins
the oracle and the CUDA path on machines where the reference tree is absent.

    make -C oracle && python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes as C
import hashlib
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
import oracle  # noqa: E402

OUT = Path(__file__).resolve().parent / "ref_vectors.npz"
SIZES = [1, 2, 3, 31, 1000, 3073, 5000, 65537]
# arrays above this size are stored as SHA-256 digests of their bytes
FULL_MAX = 5000
SEED = 0


def p(a):
    return C.c_void_p(a.ctypes.data)


def main() -> None:
    ref = oracle.ref()
    if ref is None:
        raise SystemExit("oracle/_ref/libparallax_ref.so not built (needs the reference tree)")
    for name in ("ref_reduce_f32", "ref_reduce_f64"):
        getattr(ref, name).restype = C.c_float if name.endswith("f32") else C.c_double
    ref.ref_reduce_i32.restype = C.c_int32
    ref.ref_reduce_i64.restype = C.c_int64
    for f in ("ref_copy_if_mod3_i32", "ref_remove_if_mod3_i32", "ref_partition_neg_i32",
              "ref_unique_i32", "ref_copy_if_gthalf_f32"):
        getattr(ref, f).restype = C.c_size_t
    out: dict[str, np.ndarray] = {}
    for n in SIZES:
        f32 = oracle.gen("f32_unit", SEED, n)
        f64 = oracle.gen("f64_unit", SEED, n)
        i32 = oracle.gen("i32_pm1000", SEED, n)
        i64 = oracle.gen("i64_full", SEED, n)
        u32 = oracle.gen("u32_full", SEED, n)
        out[f"reduce_f32_{n}"] = np.array([ref.ref_reduce_f32(p(f32), n)], np.float32)
        out[f"reduce_f64_{n}"] = np.array([ref.ref_reduce_f64(p(f64), n)], np.float64)
        out[f"reduce_i32_{n}"] = np.array([ref.ref_reduce_i32(p(i32), n)], np.int32)
        out[f"reduce_i64_{n}"] = np.array([ref.ref_reduce_i64(p(i64), n)], np.int64)
        for nm, x in (("i32", i32), ("i64", i64)):
            y = np.empty_like(x)
            getattr(ref, f"ref_inclusive_scan_{nm}")(p(x), p(y), n)
            out[f"inclusive_scan_{nm}_{n}"] = y
            z = np.empty_like(x)
            init = x.dtype.type(7)
            getattr(ref, f"ref_exclusive_scan_{nm}")(p(x), p(z), n,
                                                     (C.c_int32 if nm == "i32" else C.c_int64)(7))
            out[f"exclusive_scan_{nm}_{n}"] = z
            del init
        y = np.empty_like(f32)
        ref.ref_inclusive_scan_f32(p(f32), p(y), n)
        out[f"inclusive_scan_f32_{n}"] = y
        for nm, x in (("u32", u32), ("i32", i32)):
            y = x.copy()
            getattr(ref, f"ref_sort_{nm}")(p(y), n)
            out[f"sort_{nm}_{n}"] = y
        y = f32.copy()
        ref.ref_sort_f32(p(y), n)
        out[f"sort_f32_{n}"] = y
        y = np.zeros_like(i32)
        k = ref.ref_copy_if_mod3_i32(p(i32), p(y), n)
        out[f"copy_if_mod3_i32_{n}"] = y[:k].copy()
        y = i32.copy()
        k = ref.ref_remove_if_mod3_i32(p(y), n)
        out[f"remove_if_mod3_i32_{n}"] = y[:k].copy()
        y = i32.copy()
        k = ref.ref_partition_neg_i32(p(y), n)
        out[f"partition_neg_i32_{n}"] = y
        out[f"partition_neg_i32_{n}_k"] = np.array([k], np.int64)
        s = np.sort(i32 // 4)  # sorted with runs of repeated values
        k = ref.ref_unique_i32(p(s), n)
        out[f"unique_i32_{n}"] = s[:k].copy()
        y = np.zeros_like(f32)
        k = ref.ref_copy_if_gthalf_f32(p(f32), p(y), n)
        out[f"copy_if_gthalf_f32_{n}"] = y[:k].copy()
    for key in list(out):
        a = out[key]
        n = int(key.split("_")[-1]) if key.split("_")[-1].isdigit() else 0
        if a.size > 1 and n > FULL_MAX:
            out[key] = np.frombuffer(hashlib.sha256(a.tobytes()).digest(), np.uint8).copy()
            out[key + "_sha256"] = np.array([1], np.int8)
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes, {len(out)} arrays)")


if __name__ == "__main__":
    main()
