"""Output formats (slime_b200/export.py): CSV, Nether coordinates, NBT and the Litematica floor
schematic. CPU tests use a stand-in predicate from the oracle; the GPU test runs the library's."""
import io

import numpy as np
import pytest

from slime_b200 import export as ex
from slime_b200.lib import RESULT_DTYPE


def results():
    r = np.zeros(3, dtype=RESULT_DTYPE)
    r[0] = (61, 16 * 5 + 8, 16 * -3 + 8, 1234 | (1024 - 40) << 20, 90, -41)
    r[1] = (60, 16 * -1 + 8, 16 * 7 + 8, 0, -9, 7)
    r[2] = (59, -29_999_992, 29_999_992, 77, -29_999_992, 29_999_992)
    return r


def test_csv_rows_and_nether():
    buf = io.StringIO()
    ex.write_csv(results(), buf)
    lines = buf.getvalue().splitlines()
    assert lines[0] == ",".join(ex.CSV_FIELDS)
    assert lines[1] == "1,61,5,-3,88,-40,1234,-40,90,-41,11,-6"
    assert lines[2] == "2,60,-1,7,-8,120,0,,-9,7,-2,0"
    # Nether: floor division by 8 (-9 -> -2, -41 -> -6), chunks: floor division by 16.
    assert ex.nether(-1) == -1 and ex.nether(-8) == -1 and ex.nether(-9) == -2 and ex.nether(15) == 1
    assert ex.coordinates_text(results()[0], nether_coords=True) == "11 -6"
    assert ex.coordinates_text(results()[1]) == "-9 7"


def test_nbt_round_trip():
    doc = {"i": ex.Int(-5), "l": 1 << 40, "s": "Grün", "c": {"n": [ex.Int(1), ex.Int(2)]},
           "e": [], "a": np.array([-1, 2, 1 << 62], dtype=np.int64), "lc": [{"Name": "x"}, {"Name": "y"}]}
    name, back = ex.read_nbt(ex.nbt_bytes(doc, "root"))
    assert name == "root"
    assert back["i"] == -5 and isinstance(back["i"], ex.Int)
    assert back["l"] == 1 << 40 and back["s"] == "Grün" and back["c"] == {"n": [1, 2]} and back["e"] == []
    assert np.array_equal(back["a"], doc["a"]) and back["lc"] == doc["lc"]


def test_bit_array_straddles_longs():
    # 3 bits per entry: entry 21 occupies bits 63..65 and straddles longs 0 and 1.
    v = np.zeros(30, dtype=np.int64)
    v[21] = 0b101
    w = ex.pack_block_states(v, 3).view(np.uint64)
    assert w[0] == np.uint64(1) << np.uint64(63) and w[1] == np.uint64(0b10)
    rng = np.random.default_rng(7)
    for bits in range(2, 9):
        vals = rng.integers(0, 1 << bits, 4099)
        assert np.array_equal(ex.unpack_block_states(ex.pack_block_states(vals, bits), bits, len(vals)), vals)


class OracleCore:
    """Stand-in for SlimeCoreB200.is_slime_batch on the CPU (the oracle's Java predicate)."""

    def is_slime_batch(self, seed, x, z):
        from oracle.oracle import python_is_slime
        return np.array([python_is_slime(seed, int(a), int(b)) for a, b in zip(x, z)], dtype=np.uint8)


def check_floor(data, seed, site):
    meta, cells = ex.read_litematica_floor(data)
    assert cells.shape == (272, 272)
    from oracle.oracle import python_is_slime
    cx, cz = int(site["center_x"]) >> 4, int(site["center_z"]) >> 4
    want = np.zeros((17, 17), dtype=np.int64)
    for dx, dz in ex.WINDOW:
        want[dz + 8, dx + 8] = python_is_slime(seed, cx + dx, cz + dz)
    assert np.array_equal(cells, np.repeat(np.repeat(want, 16, 0), 16, 1))
    assert meta["TotalBlocks"] == 256 * int(want.sum())
    assert f"({16 * (cx - 8)}, -64, {16 * (cz - 8)})" in meta["Description"]
    return int(want.sum())


def test_litematica_floor_cpu():
    seed = 20241203
    site = results()[1]
    data = ex.litematica_floor(OracleCore(), seed, site)
    assert data[:2] == b"\x1f\x8b"
    _, root = ex.read_nbt(data)
    assert root["Version"] == ex.LITEMATICA_VERSION
    (region,) = root["Regions"].values()
    assert region["BlockStatePalette"] == [{"Name": "minecraft:air"}, {"Name": "minecraft:stone"}]
    check_floor(data, seed, site)


@pytest.mark.gpu
def test_litematica_floor_of_a_ranked_site_gpu():
    """The floor of the best site of a real search holds exactly `size` slime chunks (the window
    count the search reported), placed where the oracle's predicate puts them."""
    from slime_b200 import build
    from slime_b200.lib import SlimeCoreB200
    build.build()
    core = SlimeCoreB200()
    seed = -6166315385447640203
    total, res = core.search(seed, 3000, 40, 221, 0, 1000, -2000, 5)
    assert total > 0
    for site in res:
        n = check_floor(ex.litematica_floor(core, seed, site), seed, site)
        assert n == int(site["size"])
