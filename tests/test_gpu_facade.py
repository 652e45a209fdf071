"""The C++ facade (Config / Manager / SimManager / Agent / Map over the C ABI) gives the same
maps as the C ABI called directly with the same inputs."""
import shutil
import struct
import subprocess
from pathlib import Path

import numpy as np
import pytest

from nanomap_b200 import _native as N
from nanomap_b200 import api as A
from nanomap_b200 import scenes as S
from oracle import oracle as O
from tests.workloads import compare_maps, plain_small_frames

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


def _read_map(path):
    b = Path(path).read_bytes()
    n = struct.unpack_from("<Q", b, 0)[0]
    off = 8
    o = np.frombuffer(b, np.int32, 3 * n, off).reshape(n, 3)
    off += 12 * n
    v = np.frombuffer(b, np.float32, 512 * n, off).reshape(n, 512)
    off += 2048 * n
    a = np.frombuffer(b, np.uint32, 16 * n, off).reshape(n, 16)
    return o.copy(), v.copy(), a.copy()


def test_facade_matches_direct_abi(ctx, tmp_path):
    import torch
    cfg_dir = tmp_path / "cfg"
    shutil.copytree(ROOT / "nanomap_b200" / "config" / "headline", cfg_dir)
    spec, scene, desc_small, frames = plain_small_frames(n=3)
    # sim grid: the small world at 0.05 m, written as an NMSIMv1 voxel list
    sim_gpu = A.SimMap(ctx, 0.05, boxes=scene.boxes, cylinders=scene.cylinders, vox_min=(0, 0, 0),
                       vox_max=(400, 400, 100))
    vox = S.voxels_from_leaves(*sim_gpu.export())
    S.write_nmsim(cfg_dir / "sim_grid.nmsim", 0.05, vox)
    # frames.bin: the small scene's clouds as xyz records (step 16)
    osen = O.Sensor.from_desc(desc_small)
    W, H, step = spec.width, spec.height, 16
    recs, poses = [], []
    for pose, ranges in frames:
        r = np.zeros((W * H, 4), np.float32)
        r[:, :3] = osen.points(ranges)
        recs.append(r)
        poses.append(list(pose.position) + list(pose.orientation))
    fb = cfg_dir / "frames.bin"
    with open(fb, "wb") as f:
        f.write(struct.pack("<4i", len(frames), W, H, step))
        f.write(np.asarray(poses, np.float32).tobytes())
        for r in recs:
            f.write(r.tobytes())
    exe = tmp_path / "facade_demo"
    subprocess.run(["g++", "-std=c++17", "-O2", f"-I{ROOT / 'include'}", str(ROOT / "tests" / "cpp" / "facade_demo.cpp"),
                    f"-L{ROOT / 'nanomap_b200'}", "-lnanomap_b200", f"-Wl,-rpath,{ROOT / 'nanomap_b200'}",
                    "-o", str(exe)], check=True)
    out = subprocess.run([str(exe), str(cfg_dir / "config.txt"), str(fb), str(tmp_path / "mgr.bin"),
                          str(tmp_path / "sim.bin"), str(tmp_path / "poses.bin"),
                          str(tmp_path / "collisions.bin")],
                         capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    assert "gpu update time per loop:" in out.stdout

    # direct C ABI with the config's parameters
    h = N.NmMapDesc()
    import ctypes as C
    cfgh = C.c_void_p()
    N.call("nm_config_load", str(cfg_dir / "config.txt").encode(), C.byref(cfgh))
    N.call("nm_config_map_desc", cfgh, C.byref(h))
    descs = []
    for k in range(2):
        d = N.NmSensorDesc()
        N.call("nm_config_sensor", cfgh, k, C.byref(d), None, 0)
        descs.append(d)
    N.call("nm_config_destroy", cfgh)
    cam = A.Sensor(ctx, descs[0])
    direct = A.Map(ctx, h)
    for (pose, _), r in zip(frames, recs):
        direct.insert_points(cam, pose, r, W, H, step, flags=N.NM_SYNC)
    errs = compare_maps(_read_map(tmp_path / "mgr.bin"), direct.export())
    assert not errs, "; ".join(errs[:5])

    # sim manager: replay the logged sensor poses through render + insert
    sensors = [cam, A.Sensor(ctx, descs[1])]
    sim_file = A.SimMap(ctx, 0.05, voxels=vox)
    b = (tmp_path / "poses.bin").read_bytes()
    cnt = struct.unpack_from("<i", b, 0)[0]
    simmap = A.Map(ctx, h)
    for i in range(cnt):
        k = struct.unpack_from("<i", b, 4 + 32 * i)[0]
        vals = struct.unpack_from("<7f", b, 8 + 32 * i)
        pose = A.Pose(vals[:3], vals[3:])
        s = sensors[k]
        r = torch.zeros(s.desc.vres, s.desc.hres, device="cuda")
        sim_file.render(s, pose, r)
        simmap.insert_ranges(s, pose, r)
    assert cnt == 4
    errs = compare_maps(_read_map(tmp_path / "sim.bin"), simmap.export())
    assert not errs, "; ".join(errs[:5])
    assert simmap.stats()["rays"] > 0

    # getAgentSimCollision (SimManager.h:141-168): the agent file's 80 observation rays and
    # 0.5 m collision distance, cast from the moved agent position plus each delta
    moved = np.array(struct.unpack_from("<3f", b, 8 + 32 * (cnt - 1)), np.float32)
    c = (tmp_path / "collisions.bin").read_bytes()
    nd = struct.unpack_from("<i", c, 0)[0]
    rays = A.observation_sphere(80)
    outcomes = []
    for i in range(nd):
        d = np.array(struct.unpack_from("<3f", c, 4 + 16 * i), np.float32)
        got = struct.unpack_from("<i", c, 16 + 16 * i)[0]
        dist = sim_file.cast_rays(np.tile(moved + d, (80, 1)), rays, 0.5)
        expect = 0 if ((dist > 0) & (dist < 0.5)).any() else 1
        assert got == expect, (d, got, dist[dist > 0])
        outcomes.append(got)
    assert nd == 75


def test_vdb_sim_grid_errors(ctx, tmp_path):
    """nm_simmap_load on .vdb paths that are not OpenVDB files, or are files of a version or
    transform the reader does not take: an error status, no sim map."""
    import ctypes as C

    from tests.vdb_files import write_vdb
    h = C.c_void_p()
    p = tmp_path / "grid.vdb"
    p.write_bytes(b"\0" * 16)
    assert N.lib().nm_simmap_load(ctx.h, str(p).encode(), C.byref(h)) == N.NM_ERR_IO
    assert b"not an OpenVDB file" in N.lib().nm_last_error()
    v = np.array([[0, 0, 0], [1, 2, 3]], np.int32)
    for name, kw in (("old", dict(version=221)), ("rot", dict(transform="RotatedAffineMap")),
                     ("half_voxel", dict(transform="UniformScaleTranslateMap",
                                         translation=(0.05, 0.0, 0.0)))):
        q = write_vdb(tmp_path / f"{name}.vdb", v, res=0.1, **kw)
        assert N.lib().nm_simmap_load(ctx.h, str(q).encode(), C.byref(h)) == N.NM_ERR_UNSUPPORTED, name
    assert not h.value
