"""Compiles every test image source here (*.cu) into an sm_100a fatbin under _build/.

Each image is one translation unit exporting parallax_entry (include/parallax/kernel_abi.h),
compiled the way a compiler targeting this runtime would embed its kernels:
    nvcc -fatbin -gencode arch=compute_100a,code=sm_100a -I include -o _build/<name>.fatbin <name>.cu
Images whose name ends in _lto also export their element function (parallax_elem) and are
compiled relocatable with LTO-IR beside the machine code, so the runtime can fuse them:
    nvcc -fatbin -rdc=true -gencode arch=compute_100a,code=[sm_100a,lto_100a] ...
Rebuilt when the source, image_common.cuh or kernel_abi.h is newer than the fatbin.

    python tests/images/build_images.py
"""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
OUT = HERE / "_build"


def fatbin(name: str) -> Path:
    return OUT / f"{name}.fatbin"


def build() -> list[Path]:
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    OUT.mkdir(exist_ok=True)
    deps = [HERE / "image_common.cuh", ROOT / "include" / "parallax" / "kernel_abi.h"]
    newest_dep = max(d.stat().st_mtime for d in deps)
    built = []
    for src in sorted(HERE.glob("*.cu")):
        out = fatbin(src.stem)
        if (not out.exists() or out.stat().st_mtime < max(src.stat().st_mtime, newest_dep)):
            code = "[sm_100a,lto_100a]" if src.stem.endswith("_lto") else "sm_100a"
            cmd = [nvcc, "-fatbin", "-gencode", f"arch=compute_100a,code={code}", "-O3",
                   *(["-rdc=true"] if src.stem.endswith("_lto") else []),
                   "-I", str(ROOT / "include"), "-o", str(out), str(src)]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
        built.append(out)
    return built


if __name__ == "__main__":
    for p in build():
        print(p)
