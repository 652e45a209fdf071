"""GPU parity of the mapping path against the CPU oracle, through the C ABI.

Labels (traversed voxel sets and hit/miss/untouched per voxel) and the integrated map
(log-odds and active bits) must be bit-identical to the oracle on the same inputs.
"""
import numpy as np
import pytest

from nanomap_b200 import _native as N
from nanomap_b200 import api as A
from oracle import oracle as O
from tests.workloads import (compare_labels, compare_maps, oracle_frame, plain_small_frames)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small():
    return plain_small_frames(n=10)


def _torch(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("rounding", [N.NM_ROUND_DOWN, N.NM_ROUND_NEAREST])
def test_labels_and_map_bit_exact_plain_small(ctx, small, rounding):
    spec, scene, desc, frames = small
    res = spec.map_res
    sensor = A.Sensor(ctx, desc)
    m = A.Map(ctx, A.map_desc(res=res, rounding=rounding, clamp_min=spec.clamp[0],
                              clamp_max=spec.clamp[1]))
    om = O.Map(res, clamp_min=spec.clamp[0], clamp_max=spec.clamp[1], rounding=rounding)
    osen = O.Sensor.from_desc(desc)
    for i, (pose, ranges) in enumerate(frames):
        m.insert_ranges(sensor, pose, _torch(ranges), flags=N.NM_DEFER_INTEGRATE)
        gl = m.export_labels()
        R, eye, mt = oracle_frame(desc, pose, res, rounding)
        om.insert(R, eye, mt, desc.log_odds_hit, desc.log_odds_miss, osen.points(ranges),
                  keep_labels=True)
        errs = compare_labels(gl, om.labels())
        assert not errs, f"frame {i}: " + "; ".join(errs[:5])
        m.integrate()
    errs = compare_maps(m.export(), om.export())
    assert not errs, "; ".join(errs[:5])
    st, ost = m.stats(), om.stats()
    assert st["visits"] == ost["visits"] and st["rays"] == ost["rays"]
    assert st["unique_voxels"] == ost["unique_voxels"]
    assert st["frames"] == len(frames) and st["error_flags"] == 0


@pytest.mark.parametrize("cut", [0, 13])
def test_xyz_records_host_and_device_inputs(ctx, small, cut):
    """insertPointCloud-style input: width*height records of `step` bytes, xyz at 0/4/8.
    Host records are staged by one copy (four frames in a row without a wait, so the staging
    buffer is reused while earlier frames run); `cut` drops the last rows so that the last
    tile row is partial."""
    spec, scene, desc, frames = small
    res = spec.map_res
    sensor = A.Sensor(ctx, desc)
    osen = O.Sensor.from_desc(desc)
    m_host = A.Map(ctx, A.map_desc(res=res))
    m_dev = A.Map(ctx, A.map_desc(res=res))
    om = O.Map(res)
    H, W = spec.height - cut, spec.width
    for i, (pose, ranges) in enumerate(frames[:4]):
        pts = osen.points(ranges)[: H * W]
        rec = np.zeros((H * W, 5), np.float32)  # step 20 bytes, like the reference's Point AoS
        rec[:, :3] = pts
        rec[:, 3] = 7.0
        m_host.insert_points(sensor, pose, rec, W, H, 20)
        m_dev.insert_points(sensor, pose, _torch(rec), W, H, 20)
        R, eye, mt = oracle_frame(desc, pose, res, 1)
        om.insert(R, eye, mt, desc.log_odds_hit, desc.log_odds_miss, pts)
    oe = om.export()
    assert not compare_maps(m_host.export(), oe)
    assert not compare_maps(m_dev.export(), oe)


def test_pipelined_host_frames_with_async_status(ctx, small):
    """Host records in page-locked memory inserted without a wait: each frame's copy runs on
    the map's copy stream while the frame before it is walked (two staging buffers used in
    turn), and each frame is followed by nm_map_status_async.  The first frame has half the
    rows, so both buffers grow between asynchronous frames.  The map equals the oracle's and
    every status shows no error bits and a leaf count that never falls."""
    import torch
    spec, scene, desc, frames = small
    res = spec.map_res
    sensor = A.Sensor(ctx, desc)
    osen = O.Sensor.from_desc(desc)
    m = A.Map(ctx, A.map_desc(res=res))
    om = O.Map(res)
    H, W = spec.height, spec.width
    stream = torch.cuda.current_stream()
    reads, keep = [], []
    for i, (pose, ranges) in enumerate(frames[:6]):
        h = H // 2 if i == 0 else H
        pts = osen.points(ranges)[: h * W]
        rec = np.zeros((h * W, 4), np.float32)
        rec[:, :3] = pts
        pinned = torch.from_numpy(rec).pin_memory()
        status = torch.zeros(2, dtype=torch.int32).pin_memory()
        keep += [pinned, status]
        m.insert_points(sensor, pose, pinned, W, h, 16, stream=stream)
        m.status_async(status, stream=stream)
        ev = torch.cuda.Event()
        ev.record(stream)
        reads.append((status, ev))
        R, eye, mt = oracle_frame(desc, pose, res, 1)
        om.insert(R, eye, mt, desc.log_odds_hit, desc.log_odds_miss, pts)
    last = 0
    for status, ev in reads:
        ev.synchronize()
        leaves, err = int(status[0]), int(status[1])
        assert err == 0 and leaves >= last and leaves > 0, (leaves, err)
        last = leaves
    torch.cuda.synchronize()
    errs = compare_maps(m.export(), om.export())
    assert not errs, "; ".join(errs[:5])


@pytest.mark.parametrize("update_mode", [N.NM_UPDATE_LABEL, N.NM_UPDATE_ACCUMULATE])
@pytest.mark.parametrize("clamp_mode", [N.NM_CLAMP_ALWAYS, N.NM_CLAMP_ON_CROSSING])
@pytest.mark.parametrize("thres", [(0.3, -0.2), (1.6, -1.1)])
def test_update_modes_and_clamp_orders(ctx, small, update_mode, clamp_mode, thres):
    """Both integration kernels under both clamp orders (Handler.cpp:99-104 clamps every
    update; SimHandler.cpp:100-110 only on a threshold crossing), with clamps that five
    frames reach.  Thresholds inside the clamp range give both orders the same map;
    thresholds outside it make them differ (values past a clamp, active bits)."""
    spec, scene, desc, frames = small
    res = spec.map_res
    sensor = A.Sensor(ctx, desc)
    osen = O.Sensor.from_desc(desc)
    kw = dict(clamp_min=-1.0, clamp_max=1.5, thres_hit=thres[0], thres_miss=thres[1])
    m = A.Map(ctx, A.map_desc(res=res, update_mode=update_mode, clamp_mode=clamp_mode, **kw))
    om = O.Map(res, update_mode=1 if update_mode == N.NM_UPDATE_ACCUMULATE else 0,
               clamp_mode=clamp_mode, **kw)
    for pose, ranges in frames[:5]:
        m.insert_ranges(sensor, pose, _torch(ranges))
        R, eye, mt = oracle_frame(desc, pose, res, 1)
        om.insert(R, eye, mt, desc.log_odds_hit, desc.log_odds_miss, osen.points(ranges))
    errs = compare_maps(m.export(), om.export())
    assert not errs, "; ".join(errs[:5])


def test_edge_points_nan_inf_zero_and_range(ctx):
    """Invalid points are dropped exactly as the oracle drops them."""
    desc = A.sensor_desc(hres=8, vres=8, max_range=2.0, explicit_log_odds=1,
                         log_odds_hit=0.85, log_odds_miss=-0.4)
    sensor = A.Sensor(ctx, desc)
    res = 0.05
    pose = A.Pose((0.05, -0.025, 0.0), (1, 0, 0, 0))
    rng = np.random.default_rng(5)
    pts = rng.normal(0, 1.0, (64, 3)).astype(np.float32)
    pts[0] = np.nan
    pts[1] = np.inf
    pts[2] = 0.0
    pts[3] = (2.0, 0.0, 0.0)     # exactly max range: dropped
    pts[4] = (1.999, 0.0, 0.0)   # end voxel leaves past max range: misses only
    pts[5] = (0.0, 0.0, 1e-9)    # below the shortest direction: dropped
    pts[6] = (-0.01, 0.0, 0.0)   # inside the eye voxel
    pts[7] = (0.0, 0.7, -0.0)    # axis-aligned
    m = A.Map(ctx, A.map_desc(res=res))
    m.insert_points(sensor, pose, pts, 8, 8, 12, flags=N.NM_SYNC)
    om = O.Map(res)
    R, eye, mt = oracle_frame(desc, pose, res, 1)
    om.insert(R, eye, mt, 0.85, -0.4, pts)
    assert not compare_maps(m.export(), om.export())
    assert m.stats()["rays"] == om.stats()["rays"]


def test_empty_and_all_invalid_frames(ctx):
    desc = A.sensor_desc(hres=4, vres=4, max_range=5.0)
    sensor = A.Sensor(ctx, desc)
    m = A.Map(ctx, A.map_desc(res=0.1))
    m.insert_points(sensor, A.Pose(), np.zeros((0, 3), np.float32), 0, 0, 12, flags=N.NM_SYNC)
    bad = np.full((16, 3), np.nan, np.float32)
    m.insert_points(sensor, A.Pose(), bad, 4, 4, 12, flags=N.NM_SYNC)
    st = m.stats()
    assert st["rays"] == 0 and st["leaf_count"] == 0 and st["error_flags"] == 0


def test_table_growth_keeps_results(ctx, small):
    """A tiny initial table grows (rehash) during the run without changing the result."""
    spec, scene, desc, frames = small
    res = 0.05
    sensor = A.Sensor(ctx, desc)
    osen = O.Sensor.from_desc(desc)
    m = A.Map(ctx, A.map_desc(res=res, initial_leaf_capacity=1024))
    om = O.Map(res)
    for pose, ranges in frames:
        m.insert_ranges(sensor, pose, _torch(ranges))
        R, eye, mt = oracle_frame(desc, pose, res, 1)
        om.insert(R, eye, mt, desc.log_odds_hit, desc.log_odds_miss, osen.points(ranges))
    st = m.stats()
    assert st["grow_count"] >= 1 and st["error_flags"] == 0
    assert not compare_maps(m.export(), om.export())


def test_repeat_runs_are_bit_identical(ctx, small):
    spec, scene, desc, frames = small
    sensor = A.Sensor(ctx, desc)
    outs = []
    for _ in range(2):
        m = A.Map(ctx, A.map_desc(res=0.05))
        for pose, ranges in frames[:3]:
            m.insert_ranges(sensor, pose, _torch(ranges))
        o, v, a = m.export()
        idx = np.lexsort((o[:, 2], o[:, 1], o[:, 0]))
        outs.append((o[idx], v[idx], a[idx]))
        m.close()
    assert all(np.array_equal(x, y) for x, y in zip(outs[0], outs[1]))


def test_bad_arguments(ctx):
    desc = A.sensor_desc(hres=4, vres=4)
    sensor = A.Sensor(ctx, desc)
    m = A.Map(ctx, A.map_desc(res=0.1))
    with pytest.raises(N.NanomapError):
        m.insert_points(sensor, A.Pose(), np.zeros((16, 3), np.float32), 4, 4, 8)
    with pytest.raises(N.NanomapError):
        m.insert_ranges(sensor, A.Pose((1e9, 0, 0), (1, 0, 0, 0)), np.ones(16, np.float32))
    with pytest.raises(N.NanomapError):
        A.Map(ctx, A.map_desc(res=0.1, max_agents=0))


def test_handles_destroyed_in_any_order(small):
    """Objects keep their context alive: destroying the context handle first leaves the map,
    sensor and sim map usable, and the last one to go frees it."""
    import torch
    spec, scene, desc, frames = small
    c2 = A.Context(0)
    sensor = A.Sensor(c2, desc)
    m = A.Map(c2, A.map_desc(res=spec.map_res))
    sim = A.SimMap(c2, spec.sim_res, boxes=scene.boxes, cylinders=scene.cylinders,
                   vox_min=scene.vox_min, vox_max=scene.vox_max)
    c2.close()
    pose, _ = frames[0]
    r = torch.zeros((desc.vres, desc.hres), device="cuda")
    sim.render(sensor, pose, r)
    m.insert_ranges(sensor, pose, r, flags=N.NM_SYNC)
    assert m.stats()["leaf_count"] > 0
    sensor.close()
    sim.close()
    m.close()


def _wide_frame(seed=3):
    """A 32x24 camera at 10 m mapped at 2 mm: max_range / res = 5000 voxels, beyond the reach
    of the traversal's shared leaf table (frames past 4000 voxels take the wide traversal)."""
    rng = np.random.default_rng(seed)
    desc = A.sensor_desc(hres=32, vres=24, hfov_deg=60.0, vfov_deg=45.0, max_range=10.0,
                         explicit_log_odds=1, log_odds_hit=0.85, log_odds_miss=-0.4)
    r = rng.uniform(0.5, 9.99, (24, 32)).astype(np.float32)
    r[rng.random(r.shape) < 0.1] = 0.0       # no return
    r[rng.random(r.shape) < 0.05] = 10.5     # beyond max range: dropped
    return desc, r


@pytest.mark.parametrize("rounding", [N.NM_ROUND_DOWN, N.NM_ROUND_NEAREST])
def test_wide_frame_labels_and_map_match_oracle(ctx, rounding):
    desc, r = _wide_frame()
    res = 0.002
    sensor = A.Sensor(ctx, desc)
    pose = A.Pose((0.31, -0.27, 1.13), (0.9, 0.1, -0.2, 0.3))
    m = A.Map(ctx, A.map_desc(res=res, rounding=rounding))
    m.insert_ranges(sensor, pose, _torch(r), flags=N.NM_DEFER_INTEGRATE)
    gl = m.export_labels()
    R, eye, mt = oracle_frame(desc, pose, res, rounding)
    assert mt >= 4000.0
    om = O.Map(res, rounding=1 if rounding == N.NM_ROUND_DOWN else 0)
    osen = O.Sensor.from_desc(desc)
    om.insert(R, eye, mt, desc.log_odds_hit, desc.log_odds_miss, osen.points(r), keep_labels=True)
    errs = compare_labels(gl, om.labels())
    assert not errs, "; ".join(errs[:5])
    m.integrate()
    errs = compare_maps(m.export(), om.export())
    assert not errs, "; ".join(errs[:5])
    st = m.stats()
    assert st["visits"] == om.stats()["visits"] and st["error_flags"] == 0


def test_tick_with_a_wide_frame_matches_solo_runs(ctx, small):
    """A one-shot tick mixing a wide frame (2 mm, 10 m) with a frame of the small camera runs
    the wide traversal for both; each plane equals its solo insert."""
    spec, scene, desc_small, frames = small
    desc, r = _wide_frame(seed=5)
    res = 0.002
    wide = A.Sensor(ctx, desc)
    # the small camera with its range cut to 0.6 m (300 voxels at 2 mm), so its frames stay
    # within the leaf code's reach and its leaf bound stays small
    cam = A.Sensor(ctx, A.sensor_desc(hres=desc_small.hres, vres=desc_small.vres,
                                      hfov_deg=desc_small.hfov_deg, vfov_deg=desc_small.vfov_deg,
                                      max_range=0.6, explicit_log_odds=1, log_odds_hit=0.85,
                                      log_odds_miss=-0.4))
    pose_w = A.Pose((0.0, 0.0, 1.0), (1.0, 0.0, 0.0, 0.0))
    pose_c, rc = frames[0]
    rw, rcam = _torch(r), _torch(np.minimum(rc, 0.5).astype(np.float32))
    m = A.Map(ctx, A.map_desc(res=res, max_agents=2))
    m.tick([(wide, pose_w, rw, 0), (cam, pose_c, rcam, 1)], flags=N.NM_DEFER_INTEGRATE)
    for plane, (s, p, rr) in enumerate([(wide, pose_w, rw), (cam, pose_c, rcam)]):
        solo = A.Map(ctx, A.map_desc(res=res))
        solo.insert_ranges(s, p, rr, flags=N.NM_DEFER_INTEGRATE)
        errs = compare_labels(m.export_labels(plane), solo.export_labels(0))
        assert not errs, f"plane {plane}: " + "; ".join(errs[:3])
        solo.close()
    m.integrate()
