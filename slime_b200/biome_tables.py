"""Generates slime_b200/csrc/biome_data.h, the constant data of the FP64 biome filter.

    python -m slime_b200.biome_tables --reference-dir <reference source tree>

The biome filter needs three kinds of data that define its results and so must be exactly the
reference's (MinecraftGPUNoise.cu, gpu_noise/):

* Noise seeds. Every octave and climate noise is seeded by XOR with the MD5 of its Minecraft name
  ("octave_-9", "minecraft:continentalness", ...): Xoroshiro's fromHashOf(name) takes the first 8
  bytes of the digest (big-endian) as the low word and the next 8 as the high word. They are
  computed here from the names; nothing is copied.
* The depth spline: a tree of 41 cubic splines over (continentalness, erosion, peaks-and-valleys,
  weirdness). The reference holds it as generated code (spline_generated.cuh, one function per
  spline); this script reads that code and keeps only its control points -- per spline the input
  coordinate, and per point the location, derivative and value (a constant or a child spline) --
  which the library evaluates with its own code.
* The biome parameter trees of each Minecraft version (gpu_noise/tables/btree*.h, data from
  cubiomes, MIT License, Copyright (c) 2020 Cubitect): per node six parameter-range indices and a
  16-bit link (first child of an inner node, biome id of a leaf), per tree the parameter ranges,
  the branching order and the subtree sizes. They are re-emitted as plain arrays with the MIT
  notice.

The output is a plain C header (no namespaces), so the CUDA library and the oracle's C restatement
include the same data; the oracle's pin against the reference's own compiled code checks it.
"""
from __future__ import annotations

import argparse
import hashlib
import re
import struct
from fractions import Fraction
from pathlib import Path

OUT = Path(__file__).resolve().parent / "csrc" / "biome_data.h"

# Tree files of the reference and the version codes that select them (mcgpu_select_modern_tree,
# MinecraftGPUNoise.cu:1785-1820): (name, first version code, family, base). Family 0 is the 1.18 /
# 1.19.2 tree shape (order 10, MinecraftGPUNoise.cu:747-788), family 1 the 1.19.4+ shape (order 6,
# :686-733); both are the same branch-and-bound search, and the library searches any order and
# depth. The 1.19.4, 1.20.6 and 1.21.4 trees differ from the 1.21.5 tree in at most 100 of ~9,100
# nodes (same parameter ranges), so they are emitted as patches of it (`base`). Version codes below
# 1180 are rejected, as the reference rejects them.
TREES = [
    ("btree18", 1180, 0, None),
    ("btree192", 1192, 0, None),
    ("btree215", 1215, 1, None),
    ("btree19", 1194, 1, "btree215"),
    ("btree20", 1206, 1, "btree215"),
    ("btree21wd", 1214, 1, "btree215"),
    ("btree262", 2602, 1, None),
]

MIT_NOTICE = """\
 * MIT License
 *
 * Copyright (c) 2020 Cubitect
 *
 * Permission is hereby granted, free of charge, to any person obtaining a copy
 * of this software and associated documentation files (the "Software"), to deal
 * in the Software without restriction, including without limitation the rights
 * to use, copy, modify, merge, publish, distribute, sublicense, and/or sell
 * copies of the Software, and to permit persons to whom the Software is
 * furnished to do so, subject to the following conditions:
 *
 * The above copyright notice and this permission notice shall be included in all
 * copies or substantial portions of the Software.
 *
 * THE SOFTWARE IS PROVIDED "AS IS", WITHOUT WARRANTY OF ANY KIND, EXPRESS OR
 * IMPLIED, INCLUDING BUT NOT LIMITED TO THE WARRANTIES OF MERCHANTABILITY,
 * FITNESS FOR A PARTICULAR PURPOSE AND NONINFRINGEMENT. IN NO EVENT SHALL THE
 * AUTHORS OR COPYRIGHT HOLDERS BE LIABLE FOR ANY CLAIM, DAMAGES OR OTHER
 * LIABILITY, WHETHER IN AN ACTION OF CONTRACT, TORT OR OTHERWISE, ARISING FROM,
 * OUT OF OR IN CONNECTION WITH THE SOFTWARE OR THE USE OR OTHER DEALINGS IN THE
 * SOFTWARE."""

# Climate noises: Minecraft resource name, first octave and octave amplitudes (the noise
# parameters of the overworld), in the slot order of the filter: shift, temperature, humidity
# (vegetation), continentalness, erosion, weirdness (ridge). The large-biomes variants differ in
# name and first octave only.
CLIMATE = [
    ("minecraft:offset", None, -3, None, [1.0, 1.0, 1.0, 0.0]),
    ("minecraft:temperature", "minecraft:temperature_large", -10, -12, [1.5, 0.0, 1.0, 0.0, 0.0, 0.0]),
    ("minecraft:vegetation", "minecraft:vegetation_large", -8, -10, [1.0, 1.0, 0.0, 0.0, 0.0, 0.0]),
    ("minecraft:continentalness", "minecraft:continentalness_large", -9, -11,
     [1.0, 1.0, 2.0, 2.0, 2.0, 1.0, 1.0, 1.0, 1.0]),
    ("minecraft:erosion", "minecraft:erosion_large", -9, -11, [1.0, 1.0, 0.0, 1.0, 1.0]),
    ("minecraft:ridge", None, -7, None, [1.0, 2.0, 1.0, 0.0, 0.0, 0.0]),
]
OCTAVE_MIN = -16  # octave names "octave_-16" .. "octave_0"


def md5_pair(name: str) -> tuple[int, int]:
    d = hashlib.md5(name.encode("utf-8")).digest()
    return int.from_bytes(d[:8], "big"), int.from_bytes(d[8:], "big")


def f32_bits(text: str) -> int:
    """Bits of the float32 nearest to a decimal literal (exact rational rounding, ties to even),
    as a C compiler converts a float literal."""
    q = Fraction(text)
    d = float(q)
    b = struct.unpack("<I", struct.pack("<f", d))[0]
    best = None
    for cand in (b - 1, b, b + 1):
        if cand < 0 or cand > 0xFFFFFFFF:
            continue
        v = struct.unpack("<f", struct.pack("<I", cand))[0]
        if v != v or v in (float("inf"), float("-inf")):
            continue
        err = abs(Fraction(v) - q)
        key = (err, cand & 1)
        if best is None or key < best[0]:
            best = (key, cand)
    return best[1]


LIT = r"-?\d+\.\d+(?:e[-+]?\d+)?f"
VAL = rf"(?:{LIT}|spline_\d+\(v\))"


def _val(text: str):
    m = re.fullmatch(r"spline_(\d+)\(v\)", text)
    if m:
        return ("child", int(m.group(1)))
    return ("const", f32_bits(text.rstrip("f")))


def parse_splines(path: Path):
    """Control points of every spline function: [(coord, [(loc_bits, der_bits, value)])]."""
    src = path.read_text()
    bodies = {}
    for m in re.finditer(r"float spline_(\d+)\(const float\* v\)\n\{(.*?)\n\}\n", src, re.S):
        bodies[int(m.group(1))] = m.group(2)
    out = []
    for idx in range(len(bodies)):
        body = bodies[idx]
        coord = int(re.search(r"const float f = v\[(\d)\];", body).group(1))
        first = re.search(rf"if \(f <= ({LIT})\) \{{\s*const float n = ({VAL});\s*"
                          rf"return n \+ ({LIT}) \* \(f - ({LIT})\);", body)
        locs = [first.group(1)]
        ders = [first.group(3)]
        vals = [first.group(2)]
        assert f32_bits(first.group(4).rstrip("f")) == f32_bits(locs[0].rstrip("f"))
        for seg in re.finditer(
                rf"const float g = ({LIT});\s*const float h = ({LIT});.*?"
                rf"const float l = ({LIT});\s*const float m = ({LIT});\s*"
                rf"const float n = ({VAL});\s*const float o = ({VAL});", body, re.S):
            g, h, l, m_, n, o = seg.groups()
            assert f32_bits(g.rstrip("f")) == f32_bits(locs[-1].rstrip("f"))
            assert f32_bits(l.rstrip("f")) == f32_bits(ders[-1].rstrip("f"))
            assert n == vals[-1]
            locs.append(h)
            ders.append(m_)
            vals.append(o)
        last = re.search(rf"\n    const float n = ({VAL});\s*return n \+ ({LIT}) \* \(f - ({LIT})\);\s*$",
                         body)
        assert last.group(1) == vals[-1], idx
        assert f32_bits(last.group(2).rstrip("f")) == f32_bits(ders[-1].rstrip("f")), idx
        assert f32_bits(last.group(3).rstrip("f")) == f32_bits(locs[-1].rstrip("f")), idx
        pts = [(f32_bits(lo.rstrip("f")), f32_bits(de.rstrip("f")), _val(va))
               for lo, de, va in zip(locs, ders, vals)]
        out.append((coord, pts))
    assert re.search(r"mcgpu_depth_spline\(const float\* v\)\s*\{ return spline_0\(v\); \}", src)
    return out


def parse_tree(path: Path, name: str):
    """(order, steps, params [(lo, hi)], nodes [u64]) of one btree table."""
    src = re.sub(r"//[^\n]*", "", path.read_text())
    order = int(re.search(rf"{name}_order\s*=\s*(\d+)", src).group(1))
    steps = [int(x) for x in re.search(rf"{name}_steps\[\]\s*=\s*\{{([^}}]*)\}}", src).group(1)
             .replace(" ", "").split(",") if x]
    pblock = re.search(rf"{name}_param\[\]\[2\]\s*=\s*\{{(.*?)\}};", src, re.S).group(1)
    params = [(int(a), int(b)) for a, b in re.findall(r"\{\s*(-?\d+)\s*,\s*(-?\d+)\s*\}", pblock)]
    nblock = re.search(rf"{name}_nodes\[\]\s*=\s*\{{(.*?)\}};", src, re.S).group(1)
    nodes = [int(x, 16) for x in re.findall(r"0x([0-9A-Fa-f]+)", nblock)]
    while steps and steps[-1] == 0:
        steps.pop()
    return order, steps, params, nodes


def generate(ref_dir: Path, out: Path = OUT) -> Path:
    noise = ref_dir / "gpu_noise"
    splines = parse_splines(noise / "spline_generated.cuh")
    lines = []
    w = lines.append
    w("/* biome_data.h -- GENERATED by slime_b200/biome_tables.py; do not edit.")
    w(" *")
    w(" * Constant data of the FP64 biome filter: noise-seed hashes (MD5 of the Minecraft noise")
    w(" * names), climate octave amplitudes, the depth spline's control points and the biome")
    w(" * parameter trees of each Minecraft version. Plain C, shared by the CUDA library and the")
    w(" * oracle's C restatement.")
    w(" *")
    w(" * The biome parameter trees (BT_* arrays) are data from cubiomes, re-emitted from the")
    w(" * reference's gpu_noise/tables/btree*.h:")
    w(" *")
    w(MIT_NOTICE)
    w(" */")
    w("#ifndef SLIME_BIOME_DATA_H")
    w("#define SLIME_BIOME_DATA_H")
    w("#include <stdint.h>")
    w("")
    w("/* MD5 of \"octave_<k>\" for k = -16..0: {low word, high word}. */")
    w("static const uint64_t BD_OCTAVE_HASH[17][2] = {")
    for k in range(17):
        lo, hi = md5_pair(f"octave_{k + OCTAVE_MIN}")
        w(f"    {{0x{lo:016x}ull, 0x{hi:016x}ull}},  /* octave_{k + OCTAVE_MIN} */")
    w("};")
    w("")
    w("/* Climate noises in filter slot order: shift, temperature, humidity, continentalness,")
    w(" * erosion, weirdness. Hash of the name (normal, large biomes), first octave (normal, large),")
    w(" * octave count and amplitudes. */")
    w("typedef struct BdClimateNoise {")
    w("    uint64_t hash[2][2];")
    w("    int32_t first_octave[2];")
    w("    int32_t octaves;")
    w("    double amp[9];")
    w("} BdClimateNoise;")
    w("static const BdClimateNoise BD_CLIMATE[6] = {")
    for name, large, omin, omin_large, amps in CLIMATE:
        h0 = md5_pair(name)
        h1 = md5_pair(large or name)
        amp = ", ".join(repr(a) for a in amps + [0.0] * (9 - len(amps)))
        w(f"    {{{{{{0x{h0[0]:016x}ull, 0x{h0[1]:016x}ull}}, {{0x{h1[0]:016x}ull, 0x{h1[1]:016x}ull}}}},")
        w(f"     {{{omin}, {omin_large if omin_large is not None else omin}}}, {len(amps)}, {{{amp}}}}},"
          f"  /* {name} */")
    w("};")
    w("")
    npts = sum(len(p) for _, p in splines)
    w("/* Depth spline: spline s reads input coord BD_SPLINE_HEAD[s][0] (0 continentalness,")
    w(" * 1 erosion, 2 peaks-and-valleys, 3 weirdness) and has BD_SPLINE_HEAD[s][2] points starting")
    w(" * at BD_SPLINE_PTS[BD_SPLINE_HEAD[s][1]]. A point is {location bits, derivative bits, value")
    w(" * bits, child}: the value is the float with those bits when child < 0, else spline `child`.")
    w(" * Spline 0 is the root. */")
    def levels(s):
        kids = [v for _, _, (k, v) in splines[s][1] if k == "child"]
        return 1 + max(levels(c) for c in kids) if kids else 0
    w(f"#define BD_SPLINES {len(splines)}")
    w(f"#define BD_SPLINE_LEVELS {levels(0)}  /* nesting depth of child splines below the root */")
    w(f"#define BD_SPLINE_POINTS {npts}")
    w("static const int32_t BD_SPLINE_HEAD[BD_SPLINES][3] = {")
    first = 0
    for s, (coord, pts) in enumerate(splines):
        w(f"    {{{coord}, {first}, {len(pts)}}},  /* {s} */")
        first += len(pts)
    w("};")
    w("static const int32_t BD_SPLINE_PTS[BD_SPLINE_POINTS][4] = {")
    for s, (coord, pts) in enumerate(splines):
        for loc, der, (kind, v) in pts:
            if kind == "const":
                w(f"    {{(int32_t)0x{loc:08x}u, (int32_t)0x{der:08x}u, (int32_t)0x{v:08x}u, -1}},")
            else:
                w(f"    {{(int32_t)0x{loc:08x}u, (int32_t)0x{der:08x}u, 0, {v}}},")
    w("};")
    w("")
    w("/* Biome parameter trees. A node word holds six 8-bit parameter-range indices (bits 0..47,")
    w(" * one per climate axis: temperature, humidity, continentalness, erosion, depth, weirdness)")
    w(" * and a 16-bit link (bits 48..63): the first child of an inner node; a leaf has 0xff in the")
    w(" * top byte and its biome id in bits 48..55. A range is {lo, hi} in units of 1e-4. Children")
    w(" * of a node at depth d are `order` nodes `steps[d]` apart; a node at depth len(steps) is a")
    w(" * leaf. A tree with a patch list is its base tree's nodes with {index, word} replaced. */")
    parsed = {}
    for name, version, family, base in TREES:
        parsed[name] = parse_tree(noise / "tables" / f"{name}.h", name)
    for name, version, family, base in TREES:
        order, steps, params, nodes = parsed[name]
        up = name.upper()
        w(f"/* {name}: version codes from {version}, family {family}"
          + (f", patches of {base}" if base else "") + " */")
        w(f"#define BT_{up}_ORDER {order}")
        w(f"#define BT_{up}_DEPTH {len(steps)}")
        w(f"#define BT_{up}_PARAMS {len(params)}")
        w(f"#define BT_{up}_NODES {len(nodes)}")
        w(f"static const int32_t BT_{up}_STEPS[{len(steps)}] = {{{', '.join(map(str, steps))}}};")
        if base:
            b_order, b_steps, b_params, b_nodes = parsed[base]
            assert (b_order, b_steps, b_params, len(b_nodes)) == (order, steps, params, len(nodes)), name
            patch = [(i, n) for i, (n, m) in enumerate(zip(nodes, b_nodes)) if n != m]
            w(f"#define BT_{up}_PATCHES {len(patch)}")
            w(f"static const uint64_t BT_{up}_PATCH[{len(patch)}][2] = {{")
            for i in range(0, len(patch), 3):
                w("    " + ", ".join(f"{{{k}, 0x{v:016x}ull}}" for k, v in patch[i:i + 3]) + ",")
            w("};")
        else:
            w(f"static const int32_t BT_{up}_PARAM[{len(params)}][2] = {{")
            for i in range(0, len(params), 6):
                w("    " + ", ".join(f"{{{a}, {b}}}" for a, b in params[i:i + 6]) + ",")
            w("};")
            w(f"static const uint64_t BT_{up}_NODE[{len(nodes)}] = {{")
            for i in range(0, len(nodes), 4):
                w("    " + ", ".join(f"0x{n:016x}ull" for n in nodes[i:i + 4]) + ",")
            w("};")
        w("")
    w("typedef struct BdTree {")
    w("    int32_t version_from;  /* smallest version code that selects this tree */")
    w("    int32_t family;")
    w("    int32_t order, depth, nparams, nnodes;")
    w("    const int32_t* steps;")
    w("    const int32_t (*param)[2];")
    w("    const uint64_t* node;          /* this tree's nodes, or its base tree's */")
    w("    int32_t npatch;                /* {index, word} replacements of the base tree's nodes */")
    w("    const uint64_t (*patch)[2];")
    w("} BdTree;")
    w(f"#define BD_TREES {len(TREES)}")
    max_nodes = max(len(parsed[n][3]) for n, *_ in TREES)
    w(f"#define BD_TREE_MAX_NODES {max_nodes}")
    w("/* Ascending version_from: the tree of a version code is the last one it reaches. */")
    w("static const BdTree BD_TREE[BD_TREES] = {")
    for name, version, family, base in sorted(TREES, key=lambda t: t[1]):
        up = name.upper()
        src = (base or name).upper()
        patch = f"BT_{up}_PATCHES, BT_{up}_PATCH" if base else "0, 0"
        w(f"    {{{version}, {family}, BT_{up}_ORDER, BT_{up}_DEPTH, BT_{up}_PARAMS, BT_{up}_NODES, "
          f"BT_{up}_STEPS, BT_{src}_PARAM, BT_{src}_NODE, {patch}}},")
    w("};")
    w("")
    w("#endif /* SLIME_BIOME_DATA_H */")
    out.write_text("\n".join(lines) + "\n")
    return out


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--reference-dir", required=True, type=Path,
                    help="the reference source tree (holds gpu_noise/)")
    ap.add_argument("--out", type=Path, default=OUT)
    a = ap.parse_args()
    print(generate(a.reference_dir, a.out))


if __name__ == "__main__":
    main()
