"""Build recipe for libparallax-runtime.so (sm_100a).

Compiles every CUDA/C++ source under csrc/ with nvcc for sm_100a and links one shared
library, lib/libparallax-runtime.so, that exports the parallax C ABI. Modules under
csrc/lto/ are compiled to LTO-IR and embedded in the library as data instead: the runtime
links them with registered images at run time (nvJitLink). Objects go to
_build/ and are rebuilt when a source or any header is newer than the object. The
serving-mix load generator (loadgen/loadgen.cpp, host C++ over the public ABI) is linked
against it as lib/libparallax-loadgen.so, and the whole-heap capture shim
(heap/heap_capture.cpp) is archived as lib/libparallax-heap.a.

    python parallax-runtime_b200/build.py [--force] [--jobs N]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB_DIR = PKG / "lib"
LIB = LIB_DIR / "libparallax-runtime.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo", *ARCH,
    "-Xcompiler", "-fPIC,-fvisibility=hidden,-Wall,-Wno-unused-function",
    "--expt-relaxed-constexpr",
    "-I", str(ROOT / "include"), "-I", str(CSRC),
]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found")
    return cand


LTO_DIR = CSRC / "lto"


def sources() -> list[Path]:
    # csrc/lto/ holds modules linked at run time (embedded as LTO-IR), not library code
    return sorted(s for s in CSRC.rglob("*.cu") if LTO_DIR not in s.parents)


def build_lto_embed(force: bool, newest_header: float) -> Path:
    """Compiles every module under csrc/lto/ to an LTO-IR fatbin for sm_100a and writes an
    object that embeds the fatbins as byte arrays (pxb_lto_<stem>, pxb_lto_<stem>_size),
    which the runtime hands to nvJitLink together with a registered image."""
    obj = BUILD / "lto_embed.o"
    srcs = sorted(LTO_DIR.glob("*.cu"))
    newest = max([newest_header, *(s.stat().st_mtime for s in srcs)])
    if not force and obj.exists() and obj.stat().st_mtime >= newest:
        return obj
    lines = ["#include <stddef.h>", "/* generated by build.py: LTO-IR fatbins of csrc/lto */"]
    for src in srcs:
        fat = BUILD / f"lto_{src.stem}.fatbin"
        cmd = [nvcc(), "-std=c++17", "-O3", "-rdc=true", "-fatbin",
               "-gencode", "arch=compute_100a,code=lto_100a", "-I", str(ROOT / "include"),
               "-o", str(fat), str(src)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
        data = fat.read_bytes()
        body = ",".join(str(b) for b in data)
        lines.append(f"__attribute__((visibility(\"hidden\"), aligned(16))) const unsigned char "
                     f"pxb_lto_{src.stem}[{len(data)}] = {{{body}}};")
        lines.append(f"__attribute__((visibility(\"hidden\"))) const size_t "
                     f"pxb_lto_{src.stem}_size = {len(data)};")
    gen = BUILD / "lto_embed.c"
    gen.write_text("\n".join(lines) + "\n")
    cmd = ["gcc", "-O0", "-fPIC", "-c", str(gen), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"lto embed compile failed:\n{r.stdout}\n{r.stderr}")
    return obj


def headers() -> list[Path]:
    hs = list(CSRC.rglob("*.cuh")) + list(CSRC.rglob("*.hpp"))
    hs += list((ROOT / "include").rglob("*.h"))
    return hs


def obj_for(src: Path) -> Path:
    rel = src.relative_to(CSRC).with_suffix(".o")
    return BUILD / str(rel).replace(os.sep, "__")


def compile_one(src: Path, newest_header: float, force: bool, extra: list[str]) -> tuple[Path, str]:
    obj = obj_for(src)
    if (not force and obj.exists() and obj.stat().st_mtime >= src.stat().st_mtime
            and obj.stat().st_mtime >= newest_header):
        return obj, ""
    cmd = [nvcc(), *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(force: bool = False, jobs: int | None = None, verbose: bool = False,
          ptxas_verbose: bool = False, defines: list[str] | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    LIB_DIR.mkdir(exist_ok=True)
    newest_header = max((h.stat().st_mtime for h in headers()), default=0.0)
    extra = ["-Xptxas", "-v"] if ptxas_verbose else []
    extra += [f"-D{d}" for d in (defines or [])]
    force = force or bool(defines)
    srcs = sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(jobs) as ex:
        results = list(ex.map(lambda s: compile_one(s, newest_header, force or ptxas_verbose, extra), srcs))
    objs = [o for o, _ in results]
    objs.append(build_lto_embed(force, newest_header))
    if verbose or ptxas_verbose:
        for o, log in results:
            if log:
                print(f"== {o.name}\n{log}", file=sys.stderr)
    if (force or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs)):
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs),
               "-Xlinker", "--no-undefined", "-lpthread", "-ldl", "-lrt"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    build_loadgen(force)
    build_heap_capture(force)
    return LIB


LOADGEN_SRC = PKG / "loadgen" / "loadgen.cpp"
LOADGEN = LIB_DIR / "libparallax-loadgen.so"


def build_loadgen(force: bool = False) -> Path:
    """The serving-mix load generator: host C++ over the public C ABI only."""
    newest = max(LOADGEN_SRC.stat().st_mtime, LIB.stat().st_mtime,
                 *(h.stat().st_mtime for h in (ROOT / "include").rglob("*.h")))
    if not force and LOADGEN.exists() and LOADGEN.stat().st_mtime >= newest:
        return LOADGEN
    tmp = LOADGEN.with_suffix(".so.tmp")
    cmd = ["g++", "-std=c++17", "-O2", "-shared", "-fPIC", "-fvisibility=hidden", "-Wall",
           "-I", str(ROOT / "include"), str(LOADGEN_SRC), "-o", str(tmp),
           "-L", str(LIB_DIR), "-lparallax-runtime", "-Wl,-rpath,$ORIGIN", "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"loadgen build failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LOADGEN)
    return LOADGEN


HEAP_SRC = PKG / "heap" / "heap_capture.cpp"
HEAP_LIB = LIB_DIR / "libparallax-heap.a"


def build_heap_capture(force: bool = False) -> Path:
    """The whole-heap capture shim: a static library a program links (before the C library)
    so that its malloc / operator new allocate from the runtime's heap pool."""
    newest = max(HEAP_SRC.stat().st_mtime, (ROOT / "include" / "parallax" / "heap_pool.h").stat().st_mtime)
    if not force and HEAP_LIB.exists() and HEAP_LIB.stat().st_mtime >= newest:
        return HEAP_LIB
    obj = BUILD / "heap_capture.o"
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-Wall", "-I", str(ROOT / "include"), "-c",
           str(HEAP_SRC), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"heap capture build failed:\n{r.stdout}\n{r.stderr}")
    tmp = HEAP_LIB.with_suffix(".a.tmp")
    if tmp.exists():
        tmp.unlink()
    r = subprocess.run(["ar", "rcs", str(tmp), str(obj)], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"ar failed:\n{r.stderr}")
    os.replace(tmp, HEAP_LIB)
    return HEAP_LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--ptxas-verbose", action="store_true")
    ap.add_argument("-D", dest="defines", action="append", default=[],
                    help="preprocessor definition for every CUDA source (forces a rebuild), "
                         "e.g. -D PXB_SCAN_VPT=5 to build a different scan tile shape")
    a = ap.parse_args()
    print(build(force=a.force, jobs=a.jobs, verbose=True, ptxas_verbose=a.ptxas_verbose,
                defines=a.defines))


if __name__ == "__main__":
    main()
