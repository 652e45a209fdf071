"""GPU parity of the voxel filter (filterCloud.cu:84-434, filter type 1) against the oracle.

The filtered rays (one per end-point voxel, at the mean or the centre of its points) and their
counts must be bit-identical to the oracle's, in voxel order; a filtered insert must leave the
same labels and map as the oracle inserting those rays.
"""
import numpy as np
import pytest

from nanomap_b200 import _native as N
from nanomap_b200 import api as A
from oracle import oracle as O
from tests.workloads import compare_labels, compare_maps, oracle_frame, plain_small_frames

pytestmark = pytest.mark.gpu

IDENTITY = np.eye(3, dtype=np.float32).reshape(-1)


@pytest.fixture(scope="module")
def small():
    return plain_small_frames(n=4)


def _torch(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _check_filter(m, sensor, desc, pose, res, rounding, pts, gpu_out, centre=False):
    R, eye, mt = oracle_frame(desc, pose, res, rounding)
    op, oc = O.voxel_filter(R, eye, res, mt, rounding, pts, centre=centre)
    gp, gc = gpu_out
    assert len(gp) == len(op), (len(gp), len(op))
    assert np.array_equal(gc, oc)
    assert np.array_equal(gp.view(np.uint32), op.view(np.uint32)), \
        f"{int((gp != op).any(axis=1).sum())} of {len(gp)} filtered points differ"
    return op, oc


@pytest.mark.parametrize("rounding", [N.NM_ROUND_DOWN, N.NM_ROUND_NEAREST])
@pytest.mark.parametrize("centre", [False, True])
def test_filter_points_bit_exact(ctx, small, rounding, centre):
    spec, scene, desc, frames = small
    for res in (spec.map_res, 0.25):
        sensor = A.Sensor(ctx, desc)
        m = A.Map(ctx, A.map_desc(res=res, rounding=rounding))
        osen = O.Sensor.from_desc(desc)
        for pose, ranges in frames:
            pts = osen.points(ranges)
            # xyz records (device) and the range image (host) must give the same rays
            g1 = m.filter_points(sensor, pose, _torch(pts), desc.hres, desc.vres, 12, centre=centre)
            op, oc = _check_filter(m, sensor, desc, pose, res, rounding, pts, g1, centre)
            g2 = m.filter_points(sensor, pose, ranges, centre=centre)
            assert np.array_equal(g2[0].view(np.uint32), g1[0].view(np.uint32))
            assert np.array_equal(g2[1], g1[1])
            assert 0 < int(oc.sum()) <= int(np.count_nonzero(ranges > 0))


@pytest.mark.parametrize("rounding", [N.NM_ROUND_DOWN, N.NM_ROUND_NEAREST])
def test_filtered_insert_labels_and_map(ctx, small, rounding):
    spec, scene, desc, frames = small
    res = spec.map_res
    sensor = A.Sensor(ctx, desc)
    m = A.Map(ctx, A.map_desc(res=res, rounding=rounding, clamp_min=spec.clamp[0],
                              clamp_max=spec.clamp[1]))
    om = O.Map(res, clamp_min=spec.clamp[0], clamp_max=spec.clamp[1], rounding=rounding)
    osen = O.Sensor.from_desc(desc)
    for i, (pose, ranges) in enumerate(frames):
        m.insert_ranges(sensor, pose, _torch(ranges), flags=N.NM_DEFER_INTEGRATE | N.NM_FILTER_MEAN)
        gl = m.export_labels()
        R, eye, mt = oracle_frame(desc, pose, res, rounding)
        fp, _ = O.voxel_filter(R, eye, res, mt, rounding, osen.points(ranges))
        om.insert(IDENTITY, eye, mt, desc.log_odds_hit, desc.log_odds_miss, fp, keep_labels=True)
        errs = compare_labels(gl, om.labels())
        assert not errs, f"frame {i}: " + "; ".join(errs[:5])
        m.integrate()
    errs = compare_maps(m.export(), om.export())
    assert not errs, "; ".join(errs[:5])
    st, ost = m.stats(), om.stats()
    assert st["rays"] == ost["rays"] and st["visits"] == ost["visits"]
    assert st["error_flags"] == 0


def test_filtered_xyz_insert_accumulate_and_tiles(ctx, small):
    """Accumulate mode, host xyz input with a 16-byte step, and a non-default tile shape."""
    spec, scene, desc, frames = small
    res = spec.map_res
    sensor = A.Sensor(ctx, desc)
    m = A.Map(ctx, A.map_desc(res=res, update_mode=N.NM_UPDATE_ACCUMULATE))
    m2 = A.Map(ctx, A.map_desc(res=res))
    m2.set_launch(32, 8, 256)
    om = O.Map(res, update_mode=1)
    om2 = O.Map(res)
    osen = O.Sensor.from_desc(desc)
    for pose, ranges in frames:
        pts = osen.points(ranges)
        rec = np.zeros((len(pts), 4), np.float32)
        rec[:, :3] = pts
        m.insert_points(sensor, pose, rec, desc.hres, desc.vres, 16, flags=N.NM_FILTER_MEAN)
        m2.insert_points(sensor, pose, rec, desc.hres, desc.vres, 16, flags=N.NM_FILTER_CENTRE)
        R, eye, mt = oracle_frame(desc, pose, res, N.NM_ROUND_DOWN)
        fp, _ = O.voxel_filter(R, eye, res, mt, N.NM_ROUND_DOWN, pts)
        om.insert(IDENTITY, eye, mt, desc.log_odds_hit, desc.log_odds_miss, fp)
        fc, _ = O.voxel_filter(R, eye, res, mt, N.NM_ROUND_DOWN, pts, centre=True)
        om2.insert(IDENTITY, eye, mt, desc.log_odds_hit, desc.log_odds_miss, fc)
    errs = compare_maps(m.export(), om.export())
    assert not errs, "; ".join(errs[:5])
    errs = compare_maps(m2.export(), om2.export())
    assert not errs, "; ".join(errs[:5])


def test_filter_edge_cases(ctx, small):
    spec, scene, desc, frames = small
    res = spec.map_res
    sensor = A.Sensor(ctx, desc)
    m = A.Map(ctx, A.map_desc(res=res))
    pose = frames[0][0]
    # no returns at all
    empty = np.zeros((desc.vres, desc.hres), np.float32)
    p, c = m.filter_points(sensor, pose, empty)
    assert len(p) == 0 and len(c) == 0
    m.insert_ranges(sensor, pose, empty, flags=N.NM_FILTER_MEAN | N.NM_SYNC)
    assert m.stats()["leaf_count"] == 0
    # every point in one voxel: one ray, count = all of them; NaN and out-of-range points drop
    n = 100000
    rng = np.random.default_rng(5)
    pts = np.empty((n, 3), np.float32)
    pts[:, 0] = 0.30 + 0.01 * rng.random(n, dtype=np.float32)
    pts[:, 1] = -0.20 + 0.01 * rng.random(n, dtype=np.float32)
    pts[:, 2] = 2.00 + 0.01 * rng.random(n, dtype=np.float32)
    pts[::997] = np.nan
    pts[5::1009] = (100.0, 0.0, 0.0)
    pts[7::1013] = 0.0
    gp, gc = m.filter_points(sensor, pose, pts, n, 1, 12)
    _check_filter(m, sensor, desc, pose, res, N.NM_ROUND_DOWN, pts, (gp, gc))
    assert len(gp) <= 8 and int(gc.sum()) <= n
    # ragged cloud size (not a multiple of a tile), unaligned records, device input
    k = 12345
    buf = np.zeros(k * 13 + 1, np.uint8)
    recs = np.ndarray((k, 3), np.float32, buffer=buf[1:], offset=0, strides=(13, 4))
    recs[:] = O.Sensor.from_desc(desc).points(frames[1][1])[:k]
    import torch
    dev = torch.from_numpy(buf).cuda()
    gp, gc = m.filter_points(sensor, pose, dev[1:], k, 1, 13)
    _check_filter(m, sensor, desc, pose, res, N.NM_ROUND_DOWN, np.array(recs), (gp, gc))
