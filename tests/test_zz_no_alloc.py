"""nm_label_frame_static: labelling a frame with no device allocation inside the call.

Some callers cannot allocate device memory while they run (real-time loops that forbid
allocation after start-up; hosts whose memory pool owns the device).  This entry point keeps
its working memory in a fixed static device array instead.  The tests call it through the C
ABI with output buffers allocated beforehand by the test, and check:
* its labels against the allocating path (nm_map_insert_ranges with NM_DEFER_INTEGRATE, then
  nm_map_export_labels), bit for bit as every label comparison in this suite, on two calls in
  a row, with the device's free memory unchanged across the second call;
* its limits: an output buffer smaller than the frame's leaves, a frame that labels more than
  32768 leaves, an oversize frame, a null pointer and a non-finite resolution.
"""
import ctypes as C

import numpy as np
import pytest

from nanomap_b200 import _native as N
from nanomap_b200 import api as A
from tests.workloads import compare_labels, plain_small_frames

pytestmark = pytest.mark.gpu


def _call(sensor, pose, ranges, res, origins, words, max_leaves, status, flags=N.NM_SYNC):
    return N.lib().nm_label_frame_static(
        sensor.h, C.byref(pose.c()), C.c_void_p(ranges.data_ptr()), C.c_float(res),
        N.NM_ROUND_DOWN, C.c_void_p(origins.data_ptr()), C.c_void_p(words.data_ptr()),
        max_leaves, C.c_void_p(status.data_ptr()), flags, None)


def _allocating_labels(ctx, sensor, pose, ranges, res):
    m = A.Map(ctx, A.map_desc(res=res, rounding=N.NM_ROUND_DOWN))
    m.insert_ranges(sensor, pose, ranges, flags=N.NM_DEFER_INTEGRATE)
    ref = m.export_labels(0)
    m.close()
    return ref


def test_static_scratch_labels_match_allocating_path(ctx):
    import torch
    spec, scene, desc, frames = plain_small_frames(n=3)
    sensor = A.Sensor(ctx, desc)
    max_leaves = 8192
    origins = torch.zeros(max_leaves * 3, dtype=torch.int32, device="cuda")
    words = torch.zeros(max_leaves * 32, dtype=torch.int32, device="cuda")
    status = torch.zeros(2, dtype=torch.int32, device="cuda")
    inputs = [(pose, torch.from_numpy(ranges).cuda()) for pose, ranges in frames[:2]]
    refs = [_allocating_labels(ctx, sensor, pose, r, spec.map_res) for pose, r in inputs]
    torch.cuda.synchronize()
    for k, ((pose, r), ref) in enumerate(zip(inputs, refs)):  # two calls share the array
        free0 = torch.cuda.mem_get_info()[0]
        rc = _call(sensor, pose, r, spec.map_res, origins, words, max_leaves, status)
        free1 = torch.cuda.mem_get_info()[0]
        assert rc == N.NM_OK, N.lib().nm_last_error()
        if k == 1:  # the first call was the warm-up that made the array resident
            assert free1 == free0, f"free device memory changed by {free0 - free1} bytes"
        st = status.cpu().numpy().view(np.uint32)
        assert st[1] == 0 and 0 < st[0] <= max_leaves
        n = int(st[0])
        got = (origins.cpu().numpy()[: 3 * n].reshape(n, 3),
               words.cpu().numpy().view(np.uint32)[: 32 * n].reshape(n, 32))
        errs = compare_labels(got, ref)
        assert not errs, "; ".join(errs[:5])
        assert n == len(ref[0])


def test_static_scratch_reports_a_short_output_buffer(ctx):
    """max_leaves = 1 on a frame of many leaves: NM_ERR_CAPACITY, the full count in status[0],
    and only the first leaf's origin and words written."""
    import torch
    spec, scene, desc, frames = plain_small_frames(n=1)
    sensor = A.Sensor(ctx, desc)
    pose, ranges = frames[0]
    r = torch.from_numpy(ranges).cuda()
    origins = torch.full((3 * 4,), -7, dtype=torch.int32, device="cuda")
    words = torch.full((32 * 4,), -7, dtype=torch.int32, device="cuda")
    status = torch.zeros(2, dtype=torch.int32, device="cuda")
    rc = _call(sensor, pose, r, spec.map_res, origins, words, 1, status)
    assert rc == N.NM_ERR_CAPACITY and b"max_leaves" in N.lib().nm_last_error()
    st = status.cpu().numpy().view(np.uint32)
    ref = _allocating_labels(ctx, sensor, pose, r, spec.map_res)
    assert st[0] == len(ref[0]) > 1 and (st[1] & 8) != 0
    o = origins.cpu().numpy()
    w = words.cpu().numpy()
    assert np.all(o[3:] == -7) and np.all(w[32:] == -7), "wrote past max_leaves"
    lookup = {tuple(int(v) for v in oo): ww for oo, ww in zip(*ref)}
    assert tuple(int(v) for v in o[:3]) in lookup
    assert np.array_equal(w[:32].view(np.uint32), lookup[tuple(int(v) for v in o[:3])])


def test_static_scratch_rejects_frames_beyond_its_leaf_limit(ctx):
    """A 640x480 camera at 0.028 m with every range at 9.9 m labels ~44 000 leaves: more
    than the 32768 the array allows, fewer than its 65536 table slots.  The allocating path
    gives the count; the static call must report NM_ERR_CAPACITY and that count."""
    import torch
    desc = A.sensor_desc(hres=640, vres=480, hfov_deg=87.0, vfov_deg=58.0, max_range=10.0)
    sensor = A.Sensor(ctx, desc)
    pose = A.Pose((0.0, 0.0, 1.0), (1.0, 0.0, 0.0, 0.0))
    res = 0.028
    r = torch.full((480, 640), 9.9, dtype=torch.float32, device="cuda")
    n_ref = len(_allocating_labels(ctx, sensor, pose, r, res)[0])
    assert 32768 < n_ref < 65536
    max_leaves = 1 << 16
    origins = torch.zeros(max_leaves * 3, dtype=torch.int32, device="cuda")
    words = torch.zeros(max_leaves * 32, dtype=torch.int32, device="cuda")
    status = torch.zeros(2, dtype=torch.int32, device="cuda")
    rc = _call(sensor, pose, r, res, origins, words, max_leaves, status)
    assert rc == N.NM_ERR_CAPACITY, N.lib().nm_last_error()
    assert b"static-scratch limit of 32768" in N.lib().nm_last_error()
    st = status.cpu().numpy().view(np.uint32)
    assert st[0] == n_ref and (st[1] & 16) != 0
    # a frame within the limit works again afterwards (the array is cleared per call)
    spec, scene, desc2, frames = plain_small_frames(n=1)
    small = A.Sensor(ctx, desc2)
    pose2, ranges2 = frames[0]
    r2 = torch.from_numpy(ranges2).cuda()
    assert _call(small, pose2, r2, spec.map_res, origins, words, max_leaves, status) == N.NM_OK
    assert status.cpu().numpy().view(np.uint32)[0] == len(
        _allocating_labels(ctx, small, pose2, r2, spec.map_res)[0])


def test_static_scratch_rejects_oversize_and_bad_arguments(ctx):
    import torch
    big = A.Sensor(ctx, A.sensor_desc(hres=4096, vres=4096, max_range=5.0))
    buf = torch.zeros(16, dtype=torch.int32, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    pose = A.Pose((0, 0, 1), (1, 0, 0, 0)).c()
    rc = N.lib().nm_label_frame_static(big.h, C.byref(pose), p, C.c_float(0.1), 1, p, p, 1, p,
                                       N.NM_SYNC, None)
    assert rc == N.NM_ERR_ARG and b"static-scratch limit" in N.lib().nm_last_error()
    small = A.Sensor(ctx, A.sensor_desc(hres=8, vres=8, max_range=5.0))
    rc = N.lib().nm_label_frame_static(small.h, C.byref(pose), None, C.c_float(0.1), 1, p, p, 1,
                                       p, 0, None)
    assert rc == N.NM_ERR_ARG
    for bad in (float("inf"), float("nan"), 0.0, -0.1):
        rc = N.lib().nm_label_frame_static(small.h, C.byref(pose), p, C.c_float(bad), 1, p, p, 1,
                                           p, N.NM_SYNC, None)
        assert rc == N.NM_ERR_ARG and b"finite" in N.lib().nm_last_error(), bad
