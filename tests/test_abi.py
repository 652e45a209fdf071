"""The C ABI library: it loads, exports every declared symbol, and its host-only math matches
the oracle bit for bit (no GPU needed)."""
import ctypes as C
import math
import subprocess

import numpy as np
import pytest

from nanomap_b200 import _native as N
from nanomap_b200 import api as A
from nanomap_b200 import scenes as S
from oracle import oracle as O


def test_library_exports_every_declared_symbol():
    L = N.lib()
    declared = N.declared_symbols()
    assert len(declared) >= 25
    assert [s for s in declared if not hasattr(L, s)] == []
    out = subprocess.run(["nm", "-D", "--defined-only", str(N.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert set(declared) <= exported


def test_abi_version():
    assert N.lib().nm_abi_version() == 1


def test_null_arguments_are_rejected():
    L = N.lib()
    assert L.nm_context_create(0, None) == N.NM_ERR_ARG
    assert L.nm_sensor_create(None, None, None) == N.NM_ERR_ARG
    assert L.nm_map_create(None, None, None) == N.NM_ERR_ARG
    assert L.nm_map_insert_ranges(None, None, None, None, 0, None) == N.NM_ERR_ARG
    assert b"null" in L.nm_last_error()


def test_context_without_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    h = C.c_void_p()
    rc = N.lib().nm_context_create(0, C.byref(h))
    assert rc == N.NM_ERR_CUDA
    assert len(N.lib().nm_last_error()) > 0
    with pytest.raises(N.NanomapError):
        A.Context(0)


def _random_poses(n, seed):
    u = S.uniform(seed, 8 * n).reshape(n, 8)
    out = []
    for row in u:
        pos = tuple(float(v) for v in (row[:3] - 0.5) * 80.0)
        q = row[3:7] - 0.5
        out.append(A.Pose(pos, tuple(float(v) for v in q)))
    return out


@pytest.mark.parametrize("rounding", [N.NM_ROUND_NEAREST, N.NM_ROUND_DOWN])
def test_frame_params_match_oracle(rounding):
    desc = A.sensor_desc(**S.sensor_desc_kwargs(S.SCENES["sim_headline"]))
    for res in (0.1, 0.05, 0.02):
        for pose in _random_poses(50, 11 + rounding):
            R, eye, mt, pm = A.frame_params(desc, pose, res, rounding)
            Ro = O.rotation(pose.orientation, list(desc.frame_transform))
            eo, mto = O.frame_setup(pose.position, res, desc.max_range, rounding)
            assert np.array_equal(R.view(np.uint32), Ro.view(np.uint32))
            assert np.array_equal(eye.view(np.uint64), eo.view(np.uint64))
            assert np.float32(mt).view(np.uint32) == np.float32(mto).view(np.uint32)
    osen = O.Sensor.from_desc(desc)
    assert np.array_equal(pm.view(np.uint32), osen.params.view(np.uint32))


def test_rounding_policy_changes_eye():
    desc = A.sensor_desc(max_range=10.0)
    pose = A.Pose((1.3, -2.7, 0.9), (1, 0, 0, 0))
    _, e_rn, _, _ = A.frame_params(desc, pose, 0.05, N.NM_ROUND_NEAREST)
    _, e_rd, _, _ = A.frame_params(desc, pose, 0.05, N.NM_ROUND_DOWN)
    assert np.all(e_rd <= e_rn)
    assert np.any(e_rd != e_rn)


def test_frame_params_reject_bad_pose():
    desc = A.sensor_desc()
    with pytest.raises(N.NanomapError) as e:
        A.frame_params(desc, A.Pose((math.nan, 0, 0), (1, 0, 0, 0)), 0.1, 0)
    assert e.value.code == N.NM_ERR_ARG
    with pytest.raises(N.NanomapError):
        A.frame_params(desc, A.Pose((0, 0, 0), (0, 0, 0, 0)), 0.1, 0)
    with pytest.raises(N.NanomapError):
        A.frame_params(desc, A.Pose((0, 0, 0), (1, 0, 0, 0)), 0.0, 0)


def test_aspect_derived_hfov_matches_reference_rule():
    # FrustumData.h:265 / Sensor.h:158-161: halfWidth = aspect * tan(vfov/2) without HFOV
    desc = A.sensor_desc(hres=640, vres=480, hfov_deg=0.0, vfov_deg=43.0)
    _, _, _, pm = A.frame_params(desc, A.Pose((0, 0, 0), (1, 0, 0, 0)), 0.1, 0)
    hh = np.float32(math.tan(math.radians(43.0) / 2))
    assert pm[1] == hh
    assert pm[0] == np.float32(np.float32(640.0 / 480.0) * hh)
