"""The cave-generator oracle (oracle/nm_oracle_cave.cpp) against hand-derived answers, and the
#cavegenconfig parser of the library (host only, no device)."""
import ctypes as C
import subprocess

import numpy as np
import pytest

from nanomap_b200 import _native as N
from nanomap_b200 import api as A
from oracle import oracle as O


def test_c_library_rand_sequence_pinned():
    """The fill draws rand() % 100 after srand(seed) (CaveGen.cpp:33-37).  glibc's generator
    (additive feedback, 128-byte state) gives 1804289383, 846930886, 1681692777 after srand(1)."""
    libc = C.CDLL(None)
    libc.srand(1)
    assert [libc.rand() for _ in range(3)] == [1804289383, 846930886, 1681692777]


@pytest.mark.parametrize("fill,expect_on", [(84, True), (83, False)])
def test_first_fill_cell_uses_first_draw(fill, expect_on):
    """The first cell of the x, y, z loops is (-Dx+8, -Dy+8, -Dz+8); the first draw after
    srand(1) is 1804289383 % 100 = 83, so it is on exactly when fill > 83."""
    c = O.Cave([20, 20, 3], 0.1, fill, 0, 4, 4, 1)
    Dx, Dy, Dz = c.dims()
    assert (Dx, Dy, Dz) == (100, 100, 15)
    c.populate()
    cells = {tuple(v) for v in c.cells()}
    assert ((-Dx + 8, -Dy + 8, -Dz + 8) in cells) == expect_on


def test_dimensions_halved_rounding_up():
    # ceil(size / res) voxels, halved with odd counts rounded up (CaveGen.cpp:17-30)
    assert O.Cave([50, 50, 3.5], 0.1, 56, 4, 4, 4, 1).dims() == (250, 250, 18)
    assert O.Cave([0.35, 1.0, 0.05], 0.1, 56, 4, 4, 4, 1).dims() == (2, 5, 1)


def test_single_cell_tiles_and_band():
    """One cell = one 8^3 leaf (512 voxels).  Its closing is itself; the band
    dilate^3 minus erode^3 of an 8^3 cube counts 1960 - 8 = 1952 voxels (the L1 ball sum:
    512 + 3*3*128 + 9*32 + 8 = 1960; the eroded cube is 2^3)."""
    c = O.Cave([20, 20, 3], 0.1, 56, 4, 4, 4, 1)
    c.set_cells([[-92, -92, -7]])
    tiles = c.voxels(shell=False)
    assert len(tiles) == 512
    # the cell's leaf is the aligned 8^3 block holding it
    assert tiles.min(0).tolist() == [-96, -96, -8] and tiles.max(0).tolist() == [-89, -89, -1]
    band = c.voxels(shell=True, half_width=3, closing=1)
    assert len(band) == 1952
    assert len(c.voxels(shell=True, half_width=1, closing=0)) == (512 + 6 * 64) - 6 ** 3


def test_two_adjacent_cells_band():
    """Two face-adjacent leaves form an 8x8x16 box: band = L1 sum of radius 3 minus the
    eroded 2x2x10 box."""
    c = O.Cave([20, 20, 3], 0.1, 56, 4, 4, 4, 1)
    c.set_cells([[-92, -92, -7], [-92, -92, 1]])
    m = lambda d: 8 if d == 0 else 2  # noqa: E731
    dims = (8, 8, 16)
    total = 0
    for dx in range(4):
        for dy in range(4 - dx):
            for dz in range(4 - dx - dy):
                w = [dims[a] if d == 0 else 2 for a, d in enumerate((dx, dy, dz))]
                total += w[0] * w[1] * w[2]
    assert len(c.voxels(shell=True)) == total - 2 * 2 * 10


def test_regions_tie_goes_to_first_in_value_order():
    """Empty fill plus floor and ceiling: two planes of equal size that do not touch
    (2*Dz = 30 is not a multiple of 8, so the ceiling is off the lattice).  getRegions meets
    the floor (z = -Dz, root key z < 0) first, so keepLargestRegion keeps the floor."""
    c = O.Cave([20, 20, 3], 0.1, 0, 0, 4, 4, 1)
    c.populate()
    c.floor_ceil()
    n, big = c.regions()
    assert n == 2 and big == 23 * 23
    c.keep_largest()
    cells = c.cells()
    assert len(cells) == 23 * 23 and set(cells[:, 2].tolist()) == {-15}


def test_smoothing_drops_ceiling_and_rules():
    """smoothMap writes a fresh grid each step: the ceiling plane set before it is gone after
    one step; a full lattice with active 26 26 (never more than 26 neighbours) keeps interior
    cells (26 neighbours = min, unchanged) and drops corner cells (7 < 26)."""
    c = O.Cave([10, 10, 3.2], 0.1, 100, 1, 26, 26, 1)
    c.populate()
    c.floor_ceil()
    Dx, Dy, Dz = c.dims()
    assert any(v[2] == Dz for v in c.cells())
    c.smooth()
    cells = {tuple(v) for v in c.cells()}
    assert not any(v[2] == Dz for v in cells)
    assert (-Dx + 8, -Dy + 8, -Dz) not in cells  # a corner: 7 neighbours


def test_cave_config_parser(tmp_path):
    p = tmp_path / "cave.txt"
    p.write_text("#cavegenconfig\nfile_out caves/map1.vdb\nmap_size 40 30 2.5\ngrid_res 0.05\n"
                 "fill_percentage 47\nsmoothing_count 6\nactive 13 12\nrandom_seed 0\nseed abc\n")
    d = A.load_cave_config(p)
    assert list(d.map_size) == [40.0, 30.0, 2.5] and d.grid_res == 0.05
    assert (d.fill_percentage, d.smoothing_count, d.active_max, d.active_min) == (47, 6, 13, 12)
    assert d.time_seed == 0 and d.file_out == b"caves/map1.vdb"
    # srand receives std::hash<std::string>("abc") stored in an int: its low 32 bits, the
    # same value a g++ program computes
    src = tmp_path / "h.cpp"
    src.write_text('#include <functional>\n#include <string>\n#include <cstdio>\n'
                   'int main(){int s = std::hash<std::string>{}(std::string("abc"));'
                   'std::printf("%u", (unsigned)s);}\n')
    exe = tmp_path / "h"
    subprocess.run(["g++", "-O1", "-o", str(exe), str(src)], check=True)
    assert d.seed == int(subprocess.run([str(exe)], capture_output=True, text=True).stdout)
    q = tmp_path / "cave2.txt"
    q.write_text("#cavegenconfig\nmap_size 10 10 2\ngrid_res 0.1\nrandom_seed 1\nseed\n")
    assert A.load_cave_config(q).time_seed == 1
    bad = tmp_path / "bad.txt"
    bad.write_text("#config\n")
    with pytest.raises(N.NanomapError):
        A.load_cave_config(bad)
