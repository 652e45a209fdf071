"""GPU parity of the simulation map (voxelisation) and simulated range images against the
CPU oracle, through the C ABI.  Both are integer / first-hit results and must be identical."""
import numpy as np
import pytest

from nanomap_b200 import _native as N
from nanomap_b200 import api as A
from nanomap_b200 import scenes as S
from oracle import oracle as O
from tests.workloads import camera_desc

pytestmark = pytest.mark.gpu


def _sorted_leaves(o, w):
    idx = np.lexsort((o[:, 2], o[:, 1], o[:, 0]))
    return o[idx], w[idx]


def _maps(ctx, name, seed=1):
    sc = S.make_scene(name, seed)
    sp = sc.spec
    g = A.SimMap(ctx, sp.sim_res, boxes=sc.boxes, cylinders=sc.cylinders, vox_min=sc.vox_min,
                 vox_max=sc.vox_max)
    o = O.SimMap(sp.sim_res, sc.vox_min, sc.vox_max, sc.boxes, sc.cylinders)
    return sc, g, o


@pytest.mark.parametrize("name", ["plain_small", "sim_headline"])
def test_voxelisation_matches_oracle(ctx, name):
    sc, g, o = _maps(ctx, name)
    gb, gn, gl = g.info()
    ob, oany = o.bbox()
    assert oany and gb == ob
    assert gn == o.count()
    go, gw = _sorted_leaves(*g.export())
    oo, ow = o.export()
    assert gl == len(oo)
    assert np.array_equal(go, oo)
    assert np.array_equal(gw, ow)


def test_voxel_list_constructor(ctx):
    rng = np.random.default_rng(3)
    vox = rng.integers(-40, 40, size=(5000, 3)).astype(np.int32)
    g = A.SimMap(ctx, 0.05, voxels=vox)
    o = O.SimMap(0.05, voxels=vox)
    go, gw = _sorted_leaves(*g.export())
    oo, ow = o.export()
    assert np.array_equal(go, oo) and np.array_equal(gw, ow)
    assert g.info()[0] == o.bbox()[0]


@pytest.mark.parametrize("collapse,compression", [(False, 0x3), (True, 0x6)])
def test_vdb_sim_grid_loads_like_its_voxels(ctx, tmp_path, collapse, compression):
    """A sim grid read from a .vdb file (nm_simmap_load) holds the file's active voxels: the
    same sim map, and the same range images, as those voxels given directly; a translation of
    whole voxels shifts them.  (The files come from the test-side writer: tests/vdb_files.py.)"""
    from tests.vdb_files import write_vdb
    sc, g, _ = _maps(ctx, "plain_small")
    res = sc.spec.sim_res
    vox = A.simmap_voxels(g)
    p = write_vdb(tmp_path / "scene.vdb", vox, res=res, collapse=collapse, compression=compression,
                  codes=(0, 6, 3))
    loaded = A.SimMap.load(ctx, p)
    assert np.array_equal(A.simmap_voxels(loaded), vox)
    assert loaded.info() == g.info()
    desc = camera_desc(sc.spec, hres=320, vres=240)
    sensor = A.Sensor(ctx, desc)
    traj = S.trajectory(sc, 3, seed=7)
    for pos, q in traj:
        a = np.zeros((240, 320), np.float32)
        b = np.zeros((240, 320), np.float32)
        g.render(sensor, A.Pose(pos, q), a)
        loaded.render(sensor, A.Pose(pos, q), b)
        assert np.array_equal(a, b)
    t = write_vdb(tmp_path / "moved.vdb", vox, res=res, transform="UniformScaleTranslateMap",
                  translation=(2 * res, -3 * res, 0.0))
    moved = A.SimMap.load(ctx, t)
    assert np.array_equal(A.simmap_voxels(moved), vox + np.array([2, -3, 0], np.int32))
    for m in (loaded, moved, g):
        m.close()
    sensor.close()


@pytest.mark.parametrize("name,n", [("plain_small", 6), ("sim_headline", 2)])
def test_render_matches_oracle(ctx, name, n):
    import torch
    sc, g, o = _maps(ctx, name)
    sp = sc.spec
    desc = camera_desc(sp, min_range=0.1)
    sensor = A.Sensor(ctx, desc)
    osen = O.Sensor.from_desc(desc)
    for pos, q in S.trajectory(sc, n, seed=9):
        pose = A.Pose(pos, q)
        out = torch.zeros(sp.height, sp.width, device="cuda")
        g.render(sensor, pose, out)
        host = np.zeros((sp.height, sp.width), np.float32)
        g.render(sensor, pose, host)
        R = O.rotation(q, list(desc.frame_transform))
        ref = o.render(osen, pos, R)
        got = out.cpu().numpy()
        assert np.array_equal(got.view(np.uint32), host.view(np.uint32))
        diff = np.nonzero(got.view(np.uint32) != ref.view(np.uint32))
        assert len(diff[0]) == 0, f"{len(diff[0])} pixels differ, e.g. {got[diff][:4]} vs {ref[diff][:4]}"
        assert (ref > 0).mean() > 0.3


def test_laser_render_matches_oracle(ctx):
    import torch
    sc, g, o = _maps(ctx, "plain_small")
    desc = A.sensor_desc(type=N.NM_SENSOR_LASER, hres=1024, vres=64, hfov_deg=360.0,
                         vfov_deg=30.0, max_range=20.0, min_range=0.2,
                         frame_transform=S.OPTICAL_TO_BODY)
    sensor = A.Sensor(ctx, desc)
    osen = O.Sensor.from_desc(desc)
    for pos, q in S.trajectory(sc, 3, seed=4):
        out = torch.zeros(64, 1024, device="cuda")
        g.render(sensor, A.Pose(pos, q), out)
        ref = o.render(osen, pos, O.rotation(q, list(desc.frame_transform)))
        assert np.array_equal(out.cpu().numpy().view(np.uint32), ref.view(np.uint32))


def test_render_outside_and_empty_maps(ctx):
    import torch
    desc = A.sensor_desc(hres=32, vres=24, hfov_deg=87, vfov_deg=58, max_range=10.0)
    sensor = A.Sensor(ctx, desc)
    empty = A.SimMap(ctx, 0.1, voxels=np.zeros((0, 3), np.int32))
    out = torch.full((24, 32), 7.0, device="cuda")
    empty.render(sensor, A.Pose((1, 2, 3), (1, 0, 0, 0)), out)
    assert float(out.abs().max()) == 0.0
    # eye far outside a small box of voxels, looking away and towards it
    vox = np.array([[i, j, k] for i in range(4) for j in range(4) for k in range(4)], np.int32)
    g = A.SimMap(ctx, 0.1, voxels=vox)
    o = O.SimMap(0.1, voxels=vox)
    osen = O.Sensor.from_desc(desc)
    for q in [(1, 0, 0, 0), (0, 0, 0, 1), (0.7071, 0, 0, 0.7071), (0.5, 0.5, 0.5, 0.5)]:
        for pos in [(-1.0, 0.2, 0.2), (0.2, 0.2, 0.2), (5.0, 5.0, 5.0)]:
            out = torch.zeros(24, 32, device="cuda")
            g.render(sensor, A.Pose(pos, q), out)
            ref = o.render(osen, pos, O.rotation(q, list(desc.frame_transform)))
            assert np.array_equal(out.cpu().numpy().view(np.uint32), ref.view(np.uint32))


def test_noise_is_seeded(ctx):
    import torch
    r = torch.full((480, 640), 3.0, device="cuda")
    a, b, c = r.clone(), r.clone(), r.clone()
    ctx.add_noise(a, 0.005, 0.02, 11)
    ctx.add_noise(b, 0.005, 0.02, 11)
    ctx.add_noise(c, 0.005, 0.02, 12)
    torch.cuda.synchronize()
    assert torch.equal(a, b) and not torch.equal(a, c)
    dropped = float((a == 0).float().mean())
    assert 0.01 < dropped < 0.03
    kept = a[a > 0] - 3.0
    assert abs(float(kept.std()) - 0.005 * 9.0) < 0.005


def test_ray_casts_match_oracle(ctx):
    """Agent observation / collision rays (SimManager.h:141-168): arbitrary origins and
    directions against the sim map, first active voxel within range, bit-identical."""
    sc, g, o = _maps(ctx, "plain_small")
    rng = np.random.default_rng(21)
    n_pos = 40
    pos = np.stack([rng.uniform(0.5, 19.5, n_pos), rng.uniform(0.5, 19.5, n_pos),
                    rng.uniform(0.3, 4.7, n_pos)], axis=1).astype(np.float32)
    sphere = A.observation_sphere(64)
    origins = np.repeat(pos, 64, axis=0)
    dirs = np.tile(sphere, (n_pos, 1))
    extra = rng.normal(size=(2000, 3)).astype(np.float32) * rng.uniform(0.1, 3.0, (2000, 1)).astype(np.float32)
    extra[::97] = 0.0  # zero-length directions give no hit
    extra[5::101, 0] = 0.0  # axis-parallel components
    origins = np.concatenate([origins, np.repeat(pos[:1], 2000, axis=0)])
    dirs = np.concatenate([dirs, extra]).astype(np.float32)
    for max_range in (0.5, 5.0, 50.0):
        gd = g.cast_rays(origins, dirs, max_range)
        od = o.cast(origins, dirs, max_range)
        assert np.array_equal(gd.view(np.uint32), od.view(np.uint32)), int((gd != od).sum())
        assert (gd <= max_range).all()
    assert (gd > 0).mean() > 0.3  # at 50 m many rays meet a box (the world has no walls)
    import torch
    td = g.cast_rays(torch.from_numpy(origins).cuda(), torch.from_numpy(dirs).cuda(), 5.0)
    assert np.array_equal(td.cpu().numpy().view(np.uint32), g.cast_rays(origins, dirs, 5.0).view(np.uint32))


def test_ray_cast_agrees_with_pixel_render(ctx):
    """A laser pixel's ray cast as an arbitrary ray gives the rendered range (laser pixels have
    unit directions, so the range limits agree)."""
    import torch
    sc, g, o = _maps(ctx, "plain_small")
    desc = A.sensor_desc(type=1, hres=64, vres=16, hfov_deg=360.0, vfov_deg=30.0, max_range=8.0,
                         frame_transform=S.OPTICAL_TO_BODY)
    sensor = A.Sensor(ctx, desc)
    pose = A.Pose((10.0, 10.0, 1.5), S.yaw_quaternion(0.3))
    r = torch.zeros((16, 64), device="cuda")
    g.render(sensor, pose, r)
    osen = O.Sensor.from_desc(desc)
    R = O.rotation(pose.orientation, list(desc.frame_transform))
    d_s = osen.points(np.ones((16, 64), np.float32))  # unit-range points = pixel directions
    d_w = (R.reshape(3, 3) @ d_s.T).T.astype(np.float32)
    cast = g.cast_rays(np.tile(np.float32(pose.position), (len(d_w), 1)), d_w, 8.0)
    rr = r.cpu().numpy().reshape(-1)
    close = np.isclose(cast, rr, rtol=1e-5, atol=1e-5)
    assert close.mean() > 0.99, close.mean()


def test_render_noisy_equals_render_then_noise(ctx):
    """nm_sim_render_noisy is nm_sim_render followed by nm_ranges_add_noise, bit for bit."""
    import torch
    sc, g, o = _maps(ctx, "sim_headline")
    spec = sc.spec
    desc = camera_desc(spec)
    sensor = A.Sensor(ctx, desc)
    for k, (p, q) in enumerate(S.trajectory(sc, 3, seed=7)):
        pose = A.Pose(p, q)
        a = torch.zeros((spec.height, spec.width), device="cuda")
        b = torch.zeros_like(a)
        g.render(sensor, pose, a)
        ctx.add_noise(a, spec.noise_coef, spec.drop, 77 + k)
        g.render_noisy(sensor, pose, b, spec.noise_coef, spec.drop, 77 + k)
        assert torch.equal(a.view(torch.int32), b.view(torch.int32))
        assert (b == 0).float().mean() > spec.drop * 0.5


def _same_maps(a, b):
    ao, av, aa = a.export()
    bo, bv, ba = b.export()
    ia = np.lexsort((ao[:, 2], ao[:, 1], ao[:, 0]))
    ib = np.lexsort((bo[:, 2], bo[:, 1], bo[:, 0]))
    return (np.array_equal(ao[ia], bo[ib]) and np.array_equal(av[ia].view(np.uint32),
                                                              bv[ib].view(np.uint32))
            and np.array_equal(aa[ia], ba[ib]))


@pytest.mark.parametrize("kind", ["camera", "camera_nearest", "odd_camera", "laser", "accumulate",
                                  "filtered"])
def test_sim_insert_equals_render_then_insert(ctx, kind):
    """nm_sim_insert (the fused render + insert in label mode; render then insert for the
    per-ray sums and the voxel filter) gives the ranges and the map of nm_sim_render_noisy
    followed by nm_map_insert_ranges."""
    import torch
    sc, g, o = _maps(ctx, "sim_headline" if kind != "laser" else "plain_small")
    spec = sc.spec
    if kind == "laser":
        desc = A.sensor_desc(type=N.NM_SENSOR_LASER, hres=1024, vres=64, hfov_deg=360.0,
                             vfov_deg=30.0, max_range=20.0, min_range=0.2,
                             frame_transform=S.OPTICAL_TO_BODY)
        H, W, res = 64, 1024, 0.05
    elif kind == "odd_camera":
        # 100 x 70 pixels: the 16 x 16 tiles overhang the image on both axes
        desc = camera_desc(spec, hres=100, vres=70)
        H, W, res = 70, 100, spec.map_res
    else:
        desc = camera_desc(spec)
        H, W, res = spec.height, spec.width, spec.map_res
    sensor = A.Sensor(ctx, desc)
    mode = N.NM_UPDATE_ACCUMULATE if kind == "accumulate" else N.NM_UPDATE_LABEL
    flags = N.NM_FILTER_MEAN if kind == "filtered" else 0
    rnd = N.NM_ROUND_NEAREST if kind == "camera_nearest" else N.NM_ROUND_DOWN
    ma = A.Map(ctx, A.map_desc(res=res, clamp_min=-2.0, clamp_max=3.5, update_mode=mode,
                               rounding=rnd))
    mb = A.Map(ctx, A.map_desc(res=res, clamp_min=-2.0, clamp_max=3.5, update_mode=mode,
                               rounding=rnd))
    for k, (p, q) in enumerate(S.trajectory(sc, 3, seed=11)):
        pose = A.Pose(p, q)
        a = torch.zeros((H, W), device="cuda")
        b = torch.zeros_like(a)
        g.render_noisy(sensor, pose, a, 0.005, 0.02, 31 + k)
        ma.insert_ranges(sensor, pose, a, flags=flags)
        g.insert(mb, sensor, pose, 0.005, 0.02, 31 + k, out=b, flags=flags)
        assert torch.equal(a.view(torch.int32), b.view(torch.int32))
    torch.cuda.synchronize()
    assert _same_maps(ma, mb)
    sa, sb = ma.stats(), mb.stats()
    assert sa["visits"] == sb["visits"] and sa["rays"] == sb["rays"] and sb["error_flags"] == 0
    # without an output image, and with a host one
    mc = A.Map(ctx, A.map_desc(res=res, clamp_min=-2.0, clamp_max=3.5, update_mode=mode,
                               rounding=rnd))
    host = np.zeros((H, W), np.float32)
    for k, (p, q) in enumerate(S.trajectory(sc, 3, seed=11)):
        g.insert(mc, sensor, A.Pose(p, q), 0.005, 0.02, 31 + k,
                 out=host if k == 2 else None, flags=flags)
    assert _same_maps(ma, mc)
    assert np.array_equal(host.view(np.uint32), b.cpu().numpy().view(np.uint32))
