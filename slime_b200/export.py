"""Output formats for ranked sites: CSV, Overworld / Nether coordinates and a Litematica floor
schematic of a site's AFK window.

The reference's frontend offers these beside its map ("copy Overworld or Nether coordinates,
export CSV results or a Litematica floor schematic"); the frontend itself is not part of the
reference tree, so the layouts here are this library's own:

- CSV: one row per site in rank order with the chunk and block coordinates of the centre, the
  count, the precise score and its Y (when scored), the best AFK spot and its Nether coordinates.
- Nether coordinates: block coordinates divided by 8, rounded down (the game's ratio).
- Litematica: a gzip-compressed NBT file (format version 6) holding one region one block high: a
  floor block under every slime chunk of the site's 221-cell window (16 x 16 blocks each), air
  elsewhere, spanning the window's 17 x 17 chunks (272 x 272 blocks). The slime chunks come from
  the library's GPU predicate (slime_b200_is_slime_batch).
"""
from __future__ import annotations

import csv
import gzip
import io
import struct
import time

import numpy as np

# The 221-cell AFK window: chunk offsets (dx, dz) with dx^2 + dz^2 <= 68.
WINDOW = [(dx, dz) for dx in range(-8, 9) for dz in range(-8, 9) if dx * dx + dz * dz <= 68]
assert len(WINDOW) == 221


def chunk_of_block(b: int) -> int:
    """Chunk coordinate of a block coordinate (floor division by 16)."""
    return b >> 4


def nether(b: int) -> int:
    """Nether block coordinate of an Overworld block coordinate (floor division by 8)."""
    return b >> 3


def decode_score(obs_count: int) -> tuple[int, int | None]:
    """(score, Y) of a result's obs_count: with a Y scan the score carries (y + 1024) << 20."""
    v = int(obs_count)
    if v >> 20:
        return v & 0xFFFFF, (v >> 20) - 1024
    return v, None


def site_rows(results: np.ndarray) -> list[dict]:
    """One dict per site, in the given (rank) order."""
    rows = []
    for rank, r in enumerate(results, start=1):
        score, y = decode_score(r["obs_count"])
        bx, bz, ax, az = (int(r[k]) for k in ("center_x", "center_z", "afk_x", "afk_z"))
        rows.append({
            "rank": rank, "size": int(r["size"]),
            "chunk_x": chunk_of_block(bx), "chunk_z": chunk_of_block(bz),
            "block_x": bx, "block_z": bz,
            "score": score, "score_y": "" if y is None else y,
            "afk_x": ax, "afk_z": az,
            "nether_x": nether(ax), "nether_z": nether(az),
        })
    return rows


CSV_FIELDS = ["rank", "size", "chunk_x", "chunk_z", "block_x", "block_z", "score", "score_y",
              "afk_x", "afk_z", "nether_x", "nether_z"]


def write_csv(results: np.ndarray, out) -> None:
    """Writes the sites as CSV to a path or a text file object."""
    def emit(f):
        w = csv.DictWriter(f, fieldnames=CSV_FIELDS, lineterminator="\n")
        w.writeheader()
        w.writerows(site_rows(results))
    if hasattr(out, "write"):
        emit(out)
    else:
        with open(out, "w", newline="") as f:
            emit(f)


def coordinates_text(result, nether_coords: bool = False) -> str:
    """The best AFK spot as the "x z" text a player pastes (Overworld or Nether)."""
    x, z = int(result["afk_x"]), int(result["afk_z"])
    return f"{nether(x)} {nether(z)}" if nether_coords else f"{x} {z}"


# ---- NBT (big-endian, as Minecraft and Litematica store it) ----------------------------------

TAG_END, TAG_INT, TAG_LONG, TAG_STRING, TAG_LIST, TAG_COMPOUND, TAG_LONG_ARRAY = 0, 3, 4, 8, 9, 10, 12


class Int(int):
    """Marks a value to be written as TAG_Int (plain Python ints are written as TAG_Long)."""


def _tag_of(v) -> int:
    if isinstance(v, Int):
        return TAG_INT
    if isinstance(v, bool):
        raise TypeError("no boolean tag")
    if isinstance(v, int):
        return TAG_LONG
    if isinstance(v, str):
        return TAG_STRING
    if isinstance(v, dict):
        return TAG_COMPOUND
    if isinstance(v, np.ndarray) and v.dtype == np.int64:
        return TAG_LONG_ARRAY
    if isinstance(v, list):
        return TAG_LIST
    raise TypeError(f"no NBT tag for {type(v).__name__}")


def _put_string(buf: io.BytesIO, s: str) -> None:
    b = s.encode("utf-8")
    buf.write(struct.pack(">H", len(b)))
    buf.write(b)


def _put_payload(buf: io.BytesIO, tag: int, v) -> None:
    if tag == TAG_INT:
        buf.write(struct.pack(">i", int(v)))
    elif tag == TAG_LONG:
        buf.write(struct.pack(">q", int(v)))
    elif tag == TAG_STRING:
        _put_string(buf, v)
    elif tag == TAG_LONG_ARRAY:
        buf.write(struct.pack(">i", len(v)))
        buf.write(v.astype(">i8").tobytes())
    elif tag == TAG_LIST:
        et = _tag_of(v[0]) if v else TAG_END
        buf.write(struct.pack(">bi", et, len(v)))
        for e in v:
            _put_payload(buf, et, e)
    elif tag == TAG_COMPOUND:
        for k, e in v.items():
            t = _tag_of(e)
            buf.write(struct.pack(">b", t))
            _put_string(buf, k)
            _put_payload(buf, t, e)
        buf.write(struct.pack(">b", TAG_END))
    else:
        raise ValueError(tag)


def nbt_bytes(root: dict, name: str = "") -> bytes:
    """An uncompressed NBT document: one named root compound."""
    buf = io.BytesIO()
    buf.write(struct.pack(">b", TAG_COMPOUND))
    _put_string(buf, name)
    _put_payload(buf, TAG_COMPOUND, root)
    return buf.getvalue()


def _get(buf: io.BytesIO, fmt: str):
    return struct.unpack(fmt, buf.read(struct.calcsize(fmt)))[0]


def _get_string(buf: io.BytesIO) -> str:
    return buf.read(_get(buf, ">H")).decode("utf-8")


def _get_payload(buf: io.BytesIO, tag: int):
    if tag == TAG_INT:
        return Int(_get(buf, ">i"))
    if tag == TAG_LONG:
        return _get(buf, ">q")
    if tag == TAG_STRING:
        return _get_string(buf)
    if tag == TAG_LONG_ARRAY:
        n = _get(buf, ">i")
        return np.frombuffer(buf.read(8 * n), dtype=">i8").astype(np.int64)
    if tag == TAG_LIST:
        et, n = _get(buf, ">b"), _get(buf, ">i")
        return [_get_payload(buf, et) for _ in range(n)]
    if tag == TAG_COMPOUND:
        out = {}
        while True:
            t = _get(buf, ">b")
            if t == TAG_END:
                return out
            k = _get_string(buf)
            out[k] = _get_payload(buf, t)
    raise ValueError(f"unsupported NBT tag {tag}")


def read_nbt(data: bytes) -> tuple[str, dict]:
    """(root name, root compound) of an NBT document (gzip-compressed or not)."""
    if data[:2] == b"\x1f\x8b":
        data = gzip.decompress(data)
    buf = io.BytesIO(data)
    if _get(buf, ">b") != TAG_COMPOUND:
        raise ValueError("root is not a compound")
    name = _get_string(buf)
    return name, _get_payload(buf, TAG_COMPOUND)


# ---- Litematica ----------------------------------------------------------------------------

LITEMATICA_VERSION = 6
DEFAULT_DATA_VERSION = 4325  # Minecraft 1.21.5


def pack_block_states(indices: np.ndarray, bits: int) -> np.ndarray:
    """Litematica's bit array: entry i occupies bits i*bits .. i*bits + bits - 1 of the long array
    (bit 0 = the least significant bit of long 0); an entry may straddle two longs."""
    n = len(indices)
    words = np.zeros((n * bits + 63) // 64, dtype=np.uint64)
    off = np.arange(n, dtype=np.int64) * bits
    idx = off >> 6
    sh = (off & 63).astype(np.uint64)
    vals = indices.astype(np.uint64)
    np.bitwise_or.at(words, idx, vals << sh)
    spill = (off & 63) + bits > 64
    if spill.any():
        np.bitwise_or.at(words, idx[spill] + 1, vals[spill] >> (np.uint64(64) - sh[spill]))
    return words.view(np.int64)


def unpack_block_states(words: np.ndarray, bits: int, n: int) -> np.ndarray:
    """Inverse of pack_block_states."""
    w = words.view(np.uint64)
    off = np.arange(n, dtype=np.int64) * bits
    idx = off >> 6
    sh = (off & 63).astype(np.uint64)
    mask = np.uint64((1 << bits) - 1)
    vals = w[idx] >> sh
    spill = (off & 63) + bits > 64
    if spill.any():
        vals[spill] |= w[idx[spill] + 1] << (np.uint64(64) - sh[spill])
    return (vals & mask).astype(np.int64)


def floor_mask(core, seed: int, result) -> np.ndarray:
    """17 x 17 booleans [dz + 8][dx + 8]: the slime chunks of the site's 221-cell window (on the
    GPU, through the library's exact predicate)."""
    cx, cz = chunk_of_block(int(result["center_x"])), chunk_of_block(int(result["center_z"]))
    xs = np.array([cx + dx for dx, dz in WINDOW], dtype=np.int64)
    zs = np.array([cz + dz for dx, dz in WINDOW], dtype=np.int64)
    slime = core.is_slime_batch(seed, xs, zs)
    m = np.zeros((17, 17), dtype=bool)
    for (dx, dz), s in zip(WINDOW, slime):
        m[dz + 8, dx + 8] = bool(s)
    return m


def litematica_floor(core, seed: int, result, y: int = -64, block: str = "minecraft:stone",
                     name: str | None = None, author: str = "slime_b200",
                     data_version: int = DEFAULT_DATA_VERSION) -> bytes:
    """A .litematic file (gzip NBT) with a one-block-high floor of `block` under every slime chunk
    of the site's AFK window. The region spans chunks cx-8..cx+8, cz-8..cz+8; its north-west
    corner is block (16 (cx - 8), y, 16 (cz - 8)), which the description states (a schematic is
    placed by the player)."""
    m = floor_mask(core, seed, result)
    cx, cz = chunk_of_block(int(result["center_x"])), chunk_of_block(int(result["center_z"]))
    sx = sz = 17 * 16
    # Block index = (y * sz + z) * sx + x; palette 0 = air, 1 = the floor block.
    cells = np.repeat(np.repeat(m, 16, axis=0), 16, axis=1).astype(np.int64)  # [z][x]
    states = cells.reshape(-1)
    bits = 2  # Litematica uses at least 2 bits per entry
    now = int(time.time() * 1000)
    x0, z0 = 16 * (cx - 8), 16 * (cz - 8)
    title = name or f"slime floor {cx},{cz}"
    region = {
        "Position": {"x": Int(0), "y": Int(0), "z": Int(0)},
        "Size": {"x": Int(sx), "y": Int(1), "z": Int(sz)},
        "BlockStatePalette": [{"Name": "minecraft:air"}, {"Name": block}],
        "BlockStates": pack_block_states(states, bits),
        "TileEntities": [], "Entities": [], "PendingBlockTicks": [], "PendingFluidTicks": [],
    }
    root = {
        "MinecraftDataVersion": Int(data_version),
        "Version": Int(LITEMATICA_VERSION),
        "SubVersion": Int(1),
        "Metadata": {
            "Name": title, "Author": author,
            "Description": (f"Floor under the {int(m.sum())} slime chunks of the AFK window of chunk "
                            f"({cx}, {cz}); place the north-west corner at block ({x0}, {y}, {z0})."),
            "RegionCount": Int(1), "TotalBlocks": Int(int(states.sum())), "TotalVolume": Int(sx * sz),
            "TimeCreated": now, "TimeModified": now,
            "EnclosingSize": {"x": Int(sx), "y": Int(1), "z": Int(sz)},
        },
        "Regions": {title: region},
    }
    return gzip.compress(nbt_bytes(root))


def read_litematica_floor(data: bytes) -> tuple[dict, np.ndarray]:
    """(metadata, [z][x] palette indices of the single one-high region) of a floor schematic."""
    _, root = read_nbt(data)
    (region,) = root["Regions"].values()
    sx, sz = region["Size"]["x"], region["Size"]["z"]
    bits = max(2, (len(region["BlockStatePalette"]) - 1).bit_length())
    states = unpack_block_states(region["BlockStates"], bits, sx * sz)
    return root["Metadata"], states.reshape(sz, sx)
