"""Prepares the reference biome module's sources for the checkers (test infrastructure only).

    python oracle/ref_biome_extract.py <reference source tree> <out dir>

Writes into <out dir> (under oracle/_ref/, git-ignored, never committed):

* src/  -- a scratch copy of the reference's gpu_noise/ module (MinecraftGPUNoise.cu, mcgpu.h,
  spline_generated.cuh, tables/*.h) with the stray trailing "\\n" text removed from the end of
  the table files (it does not compile); oracle/Makefile builds the reference biome library for
  sm_100a from it, unchanged otherwise.
* ref_noise_host.inc -- the device-side math of MinecraftGPUNoise.cu (Xoroshiro, Perlin, octave
  and climate sampling, depth spline, parameter-tree search, slime test) with every __global__
  kernel and every host API function removed, for a host build (oracle/ref_biome_host.cpp
  includes it with the CUDA qualifiers defined away).

The reference tree is read where it lies and is never modified.
"""
from __future__ import annotations

import re
import shutil
import sys
from pathlib import Path


def strip_trailing_escape(text: str) -> str:
    t = text.rstrip()
    while t.endswith("\\n"):
        t = t[:-2].rstrip()
    return t + "\n"


def drop_global_functions(src: str) -> str:
    """Removes every `__global__ ... { ... }` definition (brace matched)."""
    out = []
    i = 0
    while True:
        j = src.find("__global__", i)
        if j < 0:
            out.append(src[i:])
            break
        out.append(src[i:j])
        k = src.index("{", j)
        depth = 0
        while True:
            c = src[k]
            if c == "{":
                depth += 1
            elif c == "}":
                depth -= 1
                if depth == 0:
                    break
            k += 1
        i = k + 1
    return "".join(out)


def main(ref_dir: Path, out_dir: Path) -> None:
    noise = ref_dir / "gpu_noise"
    src_dir = out_dir / "src"
    (src_dir / "tables").mkdir(parents=True, exist_ok=True)
    for name in ("MinecraftGPUNoise.cu", "mcgpu.h", "spline_generated.cuh"):
        shutil.copyfile(noise / name, src_dir / name)
    for t in sorted((noise / "tables").glob("*.h")):
        (src_dir / "tables" / t.name).write_text(strip_trailing_escape(t.read_text()))

    src = (noise / "MinecraftGPUNoise.cu").read_text()
    cut = src.index('extern "C"')
    body = drop_global_functions(src[:cut])
    body = re.sub(r'#include\s*<cuda_runtime\.h>\s*\n', "", body)
    body = body.replace('#include "mcgpu.h"', '#include "src/mcgpu.h"')
    body = body.replace('#include "spline_generated.cuh"', '#include "src/spline_generated.cuh"')
    body = re.sub(r'#include "tables/', '#include "src/tables/', body)
    (out_dir / "ref_noise_host.inc").write_text(body)


if __name__ == "__main__":
    main(Path(sys.argv[1]), Path(sys.argv[2]))
