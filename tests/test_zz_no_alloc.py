"""nm_label_frame_static: labelling a frame with no device allocation inside the call.

Some callers cannot allocate device memory while they run (real-time loops that forbid
allocation after start-up; hosts whose memory pool owns the device).  This entry point keeps
its working memory in a fixed static device array instead.  The test calls it through the C
ABI twice in a row, with output buffers allocated beforehand by the test, and checks its
labels against the allocating path (nm_map_insert_ranges with NM_DEFER_INTEGRATE, then
nm_map_export_labels), bit for bit as every label comparison in this suite.
"""
import ctypes as C

import numpy as np
import pytest

from nanomap_b200 import _native as N
from nanomap_b200 import api as A
from tests.workloads import compare_labels, plain_small_frames

pytestmark = pytest.mark.gpu


def test_static_scratch_labels_match_allocating_path(ctx):
    import torch
    spec, scene, desc, frames = plain_small_frames(n=3)
    sensor = A.Sensor(ctx, desc)
    max_leaves = 8192
    origins = torch.zeros(max_leaves * 3, dtype=torch.int32, device="cuda")
    words = torch.zeros(max_leaves * 32, dtype=torch.int32, device="cuda")
    status = torch.zeros(2, dtype=torch.int32, device="cuda")
    for pose, ranges in frames[:2]:  # two calls in a row share the static array
        r = torch.from_numpy(ranges).cuda()
        rc = N.lib().nm_label_frame_static(
            sensor.h, C.byref(pose.c()), C.c_void_p(r.data_ptr()), C.c_float(spec.map_res),
            N.NM_ROUND_DOWN, C.c_void_p(origins.data_ptr()), C.c_void_p(words.data_ptr()),
            max_leaves, C.c_void_p(status.data_ptr()), N.NM_SYNC, None)
        assert rc == N.NM_OK, N.lib().nm_last_error()
        st = status.cpu().numpy().view(np.uint32)
        assert st[1] == 0 and 0 < st[0] <= max_leaves
        n = int(st[0])
        got = (origins.cpu().numpy()[: 3 * n].reshape(n, 3),
               words.cpu().numpy().view(np.uint32)[: 32 * n].reshape(n, 32))
        m = A.Map(ctx, A.map_desc(res=spec.map_res, rounding=N.NM_ROUND_DOWN))
        m.insert_ranges(sensor, pose, r, flags=N.NM_DEFER_INTEGRATE)
        ref = m.export_labels(0)
        m.close()
        errs = compare_labels(got, ref)
        assert not errs, "; ".join(errs[:5])
        assert n == len(ref[0])


def test_static_scratch_rejects_oversize_and_bad_arguments(ctx):
    import torch
    big = A.Sensor(ctx, A.sensor_desc(hres=4096, vres=4096, max_range=5.0))
    buf = torch.zeros(16, dtype=torch.int32, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    rc = N.lib().nm_label_frame_static(big.h, C.byref(A.Pose((0, 0, 1), (1, 0, 0, 0)).c()), p,
                                       C.c_float(0.1), 1, p, p, 1, p, N.NM_SYNC, None)
    assert rc == N.NM_ERR_ARG and b"static-scratch limit" in N.lib().nm_last_error()
    small = A.Sensor(ctx, A.sensor_desc(hres=8, vres=8, max_range=5.0))
    rc = N.lib().nm_label_frame_static(small.h, C.byref(A.Pose((0, 0, 1), (1, 0, 0, 0)).c()), None,
                                       C.c_float(0.1), 1, p, p, 1, p, 0, None)
    assert rc == N.NM_ERR_ARG
