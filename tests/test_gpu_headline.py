"""Bit-exact parity at the headline size: 640x480 range frames of the 40 x 40 x 10 m scene,
10 m range, 0.05 m voxels (about 17 M voxel visits per frame), simulated and noised on the GPU
and inserted by the GPU and by the oracle (multi-threaded) from the same ranges."""
import os

import numpy as np
import pytest

from nanomap_b200 import _native as N
from nanomap_b200 import api as A
from nanomap_b200 import scenes as S
from oracle import oracle as O
from tests.workloads import compare_labels, compare_maps, oracle_frame

pytestmark = pytest.mark.gpu

THREADS = max(1, min(16, os.cpu_count() or 1))


@pytest.fixture(scope="module")
def headline(ctx):
    import torch
    spec = S.SCENES["sim_headline"]
    scene = S.make_scene(spec, 1)
    traj = S.trajectory(scene, 4, seed=7)
    desc = A.sensor_desc(**S.sensor_desc_kwargs(spec))
    sensor = A.Sensor(ctx, desc)
    sim = A.SimMap(ctx, spec.sim_res, boxes=scene.boxes, cylinders=scene.cylinders,
                   vox_min=scene.vox_min, vox_max=scene.vox_max)
    frames = []
    for k, (p, q) in enumerate(traj):
        r = torch.zeros(spec.height, spec.width, device="cuda")
        pose = A.Pose(p, q)
        sim.render(sensor, pose, r)
        ctx.add_noise(r, spec.noise_coef, spec.drop, 1000003 * (k + 1))
        frames.append((pose, r))
    torch.cuda.synchronize()
    return spec, desc, sensor, frames


def test_headline_frames_bit_exact(headline):
    spec, desc, sensor, frames = headline
    res = spec.map_res
    m = A.Map(ctx_of(sensor), A.map_desc(res=res, clamp_min=spec.clamp[0], clamp_max=spec.clamp[1]))
    om = O.Map(res, clamp_min=spec.clamp[0], clamp_max=spec.clamp[1], rounding=1)
    osen = O.Sensor.from_desc(desc)
    total = 0
    for i, (pose, r) in enumerate(frames):
        m.insert_ranges(sensor, pose, r, flags=N.NM_DEFER_INTEGRATE)
        gl = m.export_labels()
        R, eye, mt = oracle_frame(desc, pose, res, 1)
        om.insert(R, eye, mt, desc.log_odds_hit, desc.log_odds_miss, osen.points(r.cpu().numpy()),
                  threads=THREADS, keep_labels=True)
        errs = compare_labels(gl, om.labels())
        assert not errs, f"frame {i}: " + "; ".join(errs[:5])
        m.integrate()
    errs = compare_maps(m.export(), om.export())
    assert not errs, "; ".join(errs[:5])
    st, ost = m.stats(), om.stats()
    assert st["visits"] == ost["visits"] and st["rays"] == ost["rays"]
    assert st["visits"] > 10_000_000 * len(frames)
    assert st["error_flags"] == 0


def test_headline_filtered_frame_bit_exact(headline):
    spec, desc, sensor, frames = headline
    res = spec.map_res
    m = A.Map(ctx_of(sensor), A.map_desc(res=res, clamp_min=spec.clamp[0], clamp_max=spec.clamp[1]))
    om = O.Map(res, clamp_min=spec.clamp[0], clamp_max=spec.clamp[1], rounding=1)
    osen = O.Sensor.from_desc(desc)
    identity = np.eye(3, dtype=np.float32).reshape(-1)
    for pose, r in frames[:2]:
        m.insert_ranges(sensor, pose, r, flags=N.NM_FILTER_MEAN)
        R, eye, mt = oracle_frame(desc, pose, res, 1)
        fp, _ = O.voxel_filter(R, eye, res, mt, 1, osen.points(r.cpu().numpy()))
        om.insert(identity, eye, mt, desc.log_odds_hit, desc.log_odds_miss, fp, threads=THREADS)
    errs = compare_maps(m.export(), om.export())
    assert not errs, "; ".join(errs[:5])


def ctx_of(sensor):
    return sensor.ctx


def test_large_frame_sampled_rays_bit_exact(ctx):
    """Config-5 size (80 x 80 x 20 m, 0.02 m voxels, 1280x720 at 15 m): 20000 seeded pixels of
    a simulated frame, inserted as xyz records by the GPU and by the oracle, give the same map
    (rays up to 750 voxels long)."""
    import torch
    spec = S.SCENES["large_fine"]
    scene = S.make_scene(spec, 1)
    (p, q), = S.trajectory(scene, 1, seed=7)
    desc = A.sensor_desc(**S.sensor_desc_kwargs(spec))
    sensor = A.Sensor(ctx, desc)
    sim = A.SimMap(ctx, spec.sim_res, boxes=scene.boxes, cylinders=scene.cylinders,
                   vox_min=scene.vox_min, vox_max=scene.vox_max)
    pose = A.Pose(p, q)
    r = torch.zeros(spec.height, spec.width, device="cuda")
    sim.render(sensor, pose, r)
    ranges = r.cpu().numpy()
    osen = O.Sensor.from_desc(desc)
    pts = osen.points(ranges)
    pick = np.random.default_rng(3).choice(len(pts), 20000, replace=False)
    sub = np.ascontiguousarray(pts[pick], dtype=np.float32)
    m = A.Map(ctx, A.map_desc(res=spec.map_res, clamp_min=spec.clamp[0], clamp_max=spec.clamp[1]))
    m.insert_points(sensor, pose, sub, len(sub), 1, 12, flags=N.NM_SYNC)
    om = O.Map(spec.map_res, clamp_min=spec.clamp[0], clamp_max=spec.clamp[1], rounding=1)
    R, eye, mt = oracle_frame(desc, pose, spec.map_res, 1)
    om.insert(R, eye, mt, desc.log_odds_hit, desc.log_odds_miss, sub, threads=THREADS)
    errs = compare_maps(m.export(), om.export())
    assert not errs, "; ".join(errs[:5])
    st, ost = m.stats(), om.stats()
    assert st["visits"] == ost["visits"] and st["visits"] > 2_000_000
