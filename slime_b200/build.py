"""Build libslime_b200.so in-tree with nvcc for sm_100a.

    python -m slime_b200.build          # or slime_b200.build.build()

All CUDA sources under csrc/ are compiled and linked into one shared library with the CUDA
runtime linked statically, so the library loads with nothing but the driver.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "libslime_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "-Xptxas", "-O3",
         "--expt-relaxed-constexpr"]
# Per-file flags. The biome filter reproduces the reference's FP64/FP32 arithmetic operation by
# operation, so neither the device nor the host compiler may contract a multiply and an add.
FILE_FLAGS = {"biome.cu": ["--fmad=false", "-Xcompiler", "-ffp-contract=off"]}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def needs_build() -> bool:
    if not LIB.exists():
        return True
    mtime = LIB.stat().st_mtime
    deps = list(CSRC.glob("*")) + list((PKG.parent / "include").glob("*.h"))
    return any(p.stat().st_mtime > mtime for p in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not needs_build():
        return LIB
    # One object per source, compiled in parallel, then one link.
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    jobs = []
    for src in sources():
        obj = objdir / (src.stem + ".o")
        cmd = [nvcc(), *ARCH, *FLAGS, *FILE_FLAGS.get(src.name, []), "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        jobs.append((obj, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
    objs = []
    for obj, p in jobs:
        _, err = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed ({p.returncode}) on {obj.stem}.cu:\n{err[-6000:]}")
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    res = subprocess.run([nvcc(), *ARCH, "-shared", "-o", str(tmp), *objs], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc link failed ({res.returncode}):\n{res.stderr[-6000:]}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
