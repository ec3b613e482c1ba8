"""Golden vectors and known-answer cases shared by the oracle (CPU) and CUDA (gpu) tests.

ref_vectors.npz holds outputs of the reference's own host fallbacks
(include/parallax/stdpar.hpp, compiled into oracle/_ref by oracle/Makefile) on seeded
inputs; make_golden.py regenerates it. Known-answer cases restate the reference's unit
tests (tests/unit/test_*.cpp in parallax-runtime).
"""
from __future__ import annotations

import hashlib
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden" / "ref_vectors.npz"
SIZES = [1, 2, 3, 31, 1000, 3073, 5000, 65537]
SEED = 0

F32_TOL = 1e-5
F64_TOL = 1e-12

_g = None


def golden() -> dict:
    global _g
    if _g is None:
        _g = dict(np.load(GOLDEN))
    return _g


def same_as_golden(key: str, got: np.ndarray) -> bool:
    g = golden()
    want = g[key]
    if key + "_sha256" in g:
        return hashlib.sha256(np.ascontiguousarray(got).tobytes()).digest() == want.tobytes()
    return got.shape == want.shape and np.array_equal(got, want)


def inputs(n: int) -> dict:
    import oracle
    return {
        "f32": oracle.gen("f32_unit", SEED, n),
        "f64": oracle.gen("f64_unit", SEED, n),
        "i32": oracle.gen("i32_pm1000", SEED, n),
        "i64": oracle.gen("i64_full", SEED, n),
        "u32": oracle.gen("u32_full", SEED, n),
    }


def unique_input(i32: np.ndarray) -> np.ndarray:
    return np.sort(i32 // 4)


# ---- known-answer cases from the reference's unit tests --------------------------------
def kat_reduce() -> tuple[np.ndarray, float]:
    """tests/unit/test_reduce.cpp:47-64: N=5000, data[i] = i % 8, sum exactly 17500."""
    x = (np.arange(5000) % 8).astype(np.float32)
    return x, 17500.0


def kat_scan() -> tuple[np.ndarray, np.ndarray]:
    """tests/unit/test_scan.cpp:46-61: 1000 ones -> [1, 2, ..., 1000]."""
    return np.ones(1000, np.float32), np.arange(1, 1001, dtype=np.float32)


def kat_sort() -> np.ndarray:
    """tests/unit/test_sort.cpp:41-50: N=1024, v = ((N-1-i) * 2654435761) % N as float."""
    n = 1024
    i = np.arange(n, dtype=np.uint64)
    v = ((np.uint64(n - 1) - i) * np.uint64(2654435761)) % np.uint64(n)
    return v.astype(np.float32)


def kat_copy_if() -> tuple[np.ndarray, int, np.ndarray]:
    """tests/unit/test_copy_if.cpp:54-74: in[i] = i even ? 0 : i, keep x > 0.5:
    kept 500, out[j] = 2j + 1."""
    i = np.arange(1000)
    x = np.where(i % 2 == 0, 0, i).astype(np.float32)
    return x, 500, (2 * np.arange(500) + 1).astype(np.float32)


def kat_relocate() -> tuple[np.ndarray, float]:
    """tests/unit/test_physptr.cpp:50-53, :116-122: 64 ones, v*2+1 through a relocated
    host pointer -> all 3.0."""
    return np.ones(64, np.float32), 3.0


# ---- segment layouts (CSR offsets) ------------------------------------------------------
def lognormal_offsets(seed: int, num_segments: int, median: float, sigma: float,
                      lo: int, hi: int) -> np.ndarray:
    """Segment lengths ~ round(lognormal(log(median), sigma)) clipped to [lo, hi], as
    num_segments + 1 uint64 CSR offsets."""
    rng = np.random.default_rng(seed)
    lens = np.rint(rng.lognormal(np.log(median), sigma, num_segments))
    lens = np.clip(lens, lo, hi).astype(np.uint64)
    return np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)


def offsets_of(lens) -> np.ndarray:
    return np.concatenate([[0], np.cumsum(np.asarray(lens, dtype=np.uint64))]).astype(np.uint64)


def segment_layouts() -> dict:
    """Named segment layouts covering empty, single-element, tile-boundary and ragged cases."""
    return {
        "one": offsets_of([5000]),
        "one_empty": offsets_of([0]),
        "all_empty": offsets_of([0] * 17),
        "ones": offsets_of([1] * 300),
        "mixed_empty": offsets_of([0, 3, 0, 0, 1024, 1, 0, 4097, 2, 0]),
        "tile_edges": offsets_of([1023, 1024, 1025, 2047, 2048, 2049, 4095, 4096, 4097, 8192,
                                  16383, 16384, 16385]),
        "big_and_small": offsets_of([1 << 20] + [7] * 100 + [300001] + [0, 1]),
        "lognormal": lognormal_offsets(11, 500, 512, 2.0, 0, 1 << 18),
        # more segments than the planner takes per chunk (256 threads x 16), ragged and
        # partly empty: the chunks' carries and a partial last chunk
        "many": offsets_of([int(v) for v in np.random.default_rng(5).integers(0, 40, 9001)]),
    }
