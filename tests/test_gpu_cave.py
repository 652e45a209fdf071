"""Device cave generator (nm_cave_*) against the oracle's restatement of CaveGen.cpp, stage by
stage: cells after each stage bit-identical, region counts equal, and the saved voxels (leaf
tiles and the level-set band) identical as sets."""
import ctypes as C

import numpy as np
import pytest

from nanomap_b200 import api as A
from nanomap_b200 import _native as N
from oracle import oracle as O

pytestmark = pytest.mark.gpu

# (name, map_size, grid_res, fill, smoothing, (active max, min), seed, 2-D, counter fill,
#  floor and ceiling)
CASES = [
    # MapGen.txt's parameters on a smaller map; ceiling off the lattice (2*Dz = 30)
    ("shipped_3d", (20.0, 20.0, 3.0), 0.1, 56, 4, (4, 4), 1, False, False, True),
    # majority rule; ceiling a face neighbour of the top plane (2*Dz = 32)
    ("majority_3d", (16.0, 12.0, 3.2), 0.1, 50, 5, (13, 13), 12345, False, False, True),
    # test2DCaveGen's stages: columns, 8-neighbour smoothing, no floor and ceiling
    ("columns_2d", (24.0, 20.0, 2.0), 0.1, 48, 5, (4, 4), 7, True, False, False),
    # counter-based device fill at 0.05 m
    ("counter_3d", (20.0, 16.0, 4.0), 0.05, 45, 4, (13, 12), 99, False, True, True),
]


def cellset(a):
    return {tuple(int(v) for v in r) for r in a}


def make(ctx, case):
    name, size, res, fill, smooth, (amax, amin), seed, mode_2d, counter, fc = case
    desc = A.cave_desc(size, res, fill, smooth, amax, amin, seed)
    g = A.Cave(ctx, desc)
    o = O.Cave(size, res, fill, smooth, amax, amin, seed)
    return g, o


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_cave_stages_match_oracle(ctx, case):
    name, size, res, fill, smooth, act, seed, mode_2d, counter, fc = case
    g, o = make(ctx, case)
    (half, cells) = g.dims()
    assert half == o.dims()
    g.populate(mode_2d=mode_2d, counter_rng=counter)
    o.populate(mode_2d=mode_2d, counter=counter)
    gc, oc = g.cells(), o.cells()
    assert len(gc) > 0
    # same cells, and both listed in OpenVDB value order
    assert np.array_equal(gc, oc), f"{name}: fill differs ({len(gc)} vs {len(oc)} cells)"
    g.smooth(mode_2d=mode_2d)
    o.smooth(mode_2d=mode_2d)
    assert np.array_equal(g.cells(), o.cells()), f"{name}: smoothing differs"
    if fc:
        g.floor_ceil()
        o.floor_ceil()
        assert np.array_equal(g.cells(), o.cells())
    assert g.regions() == o.regions()
    g.keep_largest()
    o.keep_largest()
    assert np.array_equal(g.cells(), o.cells()), f"{name}: largest region differs"
    for shell in (False, True):
        sm = g.simmap(shell=shell)
        gv = A.simmap_voxels(sm)
        ov = o.voxels(shell=shell)
        assert len(gv) == len(ov) and np.array_equal(gv, ov), \
            f"{name} shell={shell}: {len(gv)} vs {len(ov)} voxels"
        _, nvox, _ = sm.info()
        assert nvox == len(ov)
        sm.close()
    g.close()


def test_cave_band_widths_match_oracle(ctx):
    case = CASES[1]
    g, o = make(ctx, case)
    g.populate()
    o.populate()
    g.smooth()
    o.smooth()
    g.keep_largest()
    o.keep_largest()
    for hw, cl in ((1, 0), (2, 2), (5, 1)):
        sm = g.simmap(shell=True, half_width=hw, closing=cl)
        assert np.array_equal(A.simmap_voxels(sm), o.voxels(True, hw, cl)), (hw, cl)
        sm.close()


def test_cave_tie_keeps_floor(ctx):
    """Floor and ceiling planes of equal size and no fill: the floor comes first in value
    order and is kept (the oracle's answer, pinned by hand in the CPU tests)."""
    g = A.Cave(ctx, A.cave_desc((20.0, 20.0, 3.0), 0.1, 0, 0, 4, 4, 1))
    g.populate()
    g.floor_ceil()
    assert g.regions() == (2, 23 * 23)
    g.keep_largest()
    c = g.cells()
    assert len(c) == 23 * 23 and set(c[:, 2].tolist()) == {-15}


def test_cave_empty_lattice(ctx):
    """A map smaller than two leaves per side has no cells: every stage runs and the sim map
    is empty."""
    g = A.Cave(ctx, A.cave_desc((1.0, 1.0, 1.0), 0.1, 56, 4, 4, 4, 1))
    assert g.dims()[1][:2] == (0, 0)
    g.populate()
    g.smooth()
    g.floor_ceil()
    assert g.regions() == (0, 0)
    g.keep_largest()
    assert len(g.cells()) == 0
    sm = g.simmap()
    assert sm.info()[1] == 0
    sm.close()


@pytest.mark.parametrize("name", ["map1.vdb", "map1.nmsim"])
def test_cave_save_and_load(ctx, tmp_path, name):
    """The cave written to the reference's file_out (a .vdb grid "grid", or an NMSIMv1 list)
    and loaded as a sim grid equals the cave's sim map."""
    g, o = make(ctx, CASES[0])
    g.populate()
    g.smooth()
    g.floor_ceil()
    g.keep_largest()
    written = g.save(tmp_path / name)
    assert written.endswith(name)
    h = C.c_void_p()
    N.call("nm_simmap_load", ctx.h, written.encode(), C.byref(h))
    loaded = A.SimMap._adopt(ctx, 0.1, h)
    sm = g.simmap()
    assert np.array_equal(A.simmap_voxels(loaded), A.simmap_voxels(sm))
    assert loaded.info() == sm.info()
    loaded.close()
    sm.close()


def test_cave_raycast_from_inside(ctx):
    """A sensor inside the kept region sees the band: every cast from a free cell centre
    along the axes hits within the map."""
    g, o = make(ctx, CASES[1])
    g.populate()
    g.smooth()
    g.floor_ceil()
    g.keep_largest()
    cells = g.cells()
    sm = g.simmap()
    res = 0.1
    # the centres of the kept cells' leaves
    centres = (((cells >> 3) * 8) + 4).astype(np.float32) * res
    dirs = np.tile(np.eye(3, dtype=np.float32), (len(centres), 1))
    origins = np.repeat(centres, 3, axis=0)
    d = sm.cast_rays(origins, dirs, 100.0)
    assert np.all(d >= 0)
    assert np.mean(d > 0) > 0.5
    sm.close()


@pytest.mark.parametrize("mode", ["3d", "2d", "gen"])
def test_cavegen_facade_program(ctx, tmp_path, mode):
    """The reference's generator mains, written against nanomap::mapgen::CaveGen, give the
    oracle's cave for the same #cavegenconfig file (seed string hashed as the reference does)."""
    import subprocess
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    cfg = tmp_path / "cave.txt"
    active = "13 13" if mode == "3d" else "4 4"
    cfg.write_text(f"#cavegenconfig\nfile_out {tmp_path / 'map1.vdb'}\nmap_size 16 12 3.2\n"
                   f"grid_res 0.1\nfill_percentage 50\nsmoothing_count 4\nactive {active}\n"
                   "random_seed 0\nseed nanomap\n")
    exe = tmp_path / "cavegen_demo"
    subprocess.run(["g++", "-std=c++17", "-O2", f"-I{root / 'include'}",
                    str(root / "tests" / "cpp" / "cavegen_demo.cpp"), f"-L{root / 'nanomap_b200'}",
                    "-lnanomap_b200", f"-Wl,-rpath,{root / 'nanomap_b200'}", "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe), str(cfg), mode], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    written, n_regions, largest = out.stdout.split()
    assert written == str(tmp_path / "map1.vdb")
    d = A.load_cave_config(cfg)
    o = O.Cave(list(d.map_size), d.grid_res, d.fill_percentage, d.smoothing_count,
               d.active_max, d.active_min, d.seed)
    if mode == "2d":
        o.populate(mode_2d=True)
        o.smooth(mode_2d=True)
    else:
        o.populate()
        o.smooth()
        if mode == "3d":
            o.floor_ceil()
    assert (int(n_regions), int(largest)) == o.regions()
    if mode != "gen":
        o.keep_largest()
    vs, tr, v = A.vdb_active_voxels(written)
    assert np.float32(vs[0]) == np.float32(0.1) and not tr.any()
    v = v[np.lexsort((v[:, 2], v[:, 1], v[:, 0]))]
    assert np.array_equal(v, o.voxels(shell=True))


@pytest.mark.parametrize("seed", [0, 1, 2**31 - 1, 2**31, 2**32 - 1, 0x9E3779B9])
@pytest.mark.parametrize("mode_2d", [False, True])
def test_cave_fill_reproduces_c_library_rand(ctx, seed, mode_2d):
    """The device draws the C library's rand() sequence after srand(seed) in the reference's
    loop order (several jump chunks: 48 x 48 columns, 3 fill planes)."""
    g = A.Cave(ctx, A.cave_desc((40.0, 40.0, 4.0), 0.1, 50, 0, 4, 4, seed))
    o = O.Cave((40.0, 40.0, 4.0), 0.1, 50, 0, 4, 4, seed)
    g.populate(mode_2d=mode_2d)
    o.populate(mode_2d=mode_2d)
    assert np.array_equal(g.cells(), o.cells())
