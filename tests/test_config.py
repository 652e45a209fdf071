"""Config files in NanoMap's formats (#config / #frustumconfig / #laserconfig / #agentconfig),
parsed through the C ABI on the host (no device needed)."""
import ctypes as C
import math
from pathlib import Path

import numpy as np
import pytest

from nanomap_b200 import _native as N

HEADLINE = Path(__file__).resolve().parents[1] / "nanomap_b200" / "config" / "headline" / "config.txt"


def load(path):
    h = C.c_void_p()
    N.call("nm_config_load", str(path).encode(), C.byref(h))
    return h


def info(h):
    i = N.NmConfigInfo()
    N.call("nm_config_get_info", h, C.byref(i))
    return i


def sensor(h, k):
    d = N.NmSensorDesc()
    name = C.create_string_buffer(256)
    N.call("nm_config_sensor", h, k, C.byref(d), name, 256)
    return name.value.decode(), d


def test_headline_config_values():
    h = load(HEADLINE)
    i = info(h)
    assert i.mapping_res == np.float32(0.05) and i.grid_res == np.float32(0.05)
    assert i.leaf_edge == 8 and i.n_sensors == 2 and i.n_agents == 1
    assert i.clamp_min == np.float32(-2.0) and i.clamp_max == np.float32(3.5)
    assert i.update_mode == N.NM_UPDATE_LABEL and i.rounding == N.NM_ROUND_DOWN
    assert i.process_type == 1  # a frustum sensor exists (Config.cpp:55-57)
    assert i.sim_grid.decode().endswith("sim_grid.nmsim")
    name, d = sensor(h, 0)
    assert name == "camera_640x480" and d.type == N.NM_SENSOR_FRUSTUM
    assert (d.hres, d.vres, d.id) == (640, 480, 2000)
    assert d.hfov_deg == 87.0 and d.vfov_deg == 58.0 and d.max_range == 10.0
    assert d.explicit_log_odds == 1 and d.log_odds_hit == np.float32(0.85) and d.log_odds_miss == np.float32(-0.4)
    assert list(d.frame_transform) == [0.0, -1.0, 0.0, 0.0, 0.0, 1.0, 1.0, 0.0, 0.0]
    name, d = sensor(h, 1)
    assert name == "spinning_64x1024" and d.type == N.NM_SENSOR_LASER
    assert (d.hres, d.vres) == (1024, 64)  # hRes = hfov/aHRes + 1 (LaserData.h:260-261)
    a = N.NmAgentInfo()
    N.call("nm_config_agent", h, 0, C.byref(a))
    assert a.spawn_random == 0 and list(a.position) == [10.0, 10.0, 1.5] and a.n_sensors == 2
    assert a.num_obs == 80 and a.len_obs == 20.0
    nm = C.create_string_buffer(64)
    p = N.NmPose()
    N.call("nm_config_agent_sensor", h, 0, 1, nm, 64, C.byref(p))
    assert nm.value == b"spinning_64x1024"
    assert list(p.position) == [0.0, 0.0, np.float32(0.3)]
    assert np.allclose(list(p.orientation), [0.9238795, 0.0, 0.0, 0.3826834])
    md = N.NmMapDesc()
    N.call("nm_config_map_desc", h, C.byref(md))
    assert md.res == np.float32(0.05) and md.thres_hit == 0.0 and md.thres_miss == 0.0
    N.call("nm_config_destroy", h)


def _write(tmp, name, text):
    p = tmp / name
    p.write_text(text)
    return p


def test_reference_style_config_and_defaults(tmp_path):
    """The reference's own key set (PublishType, no extension keys): defaults apply."""
    _write(tmp_path, "cam.txt", "#frustumconfig\nName:\ncam\nId:\n7\nHRes:\n640\nVRes:\n480\nVFOV:\n43\n"
           "Rate:\n50\nMaxRange:\n10\nMinRange:\n0.1\nProbHit:\n0.95\nProbMiss:\n0.3\n"
           "FrameTransform:\n0.0 -1.0 0.0\n0.0 0.0 1.0\n1.0 0.0 0.0\n#endconfig\n")
    _write(tmp_path, "vlp.txt", "#laserconfig\nName:\nVLP16\nId:\n1001\nAngularHRes:\n0.4\nAngularVRes:\n2\n"
           "HFOV:\n360\nVFOV:\n30\nRate:\n20\nMaxRange:\n50\nMinRange:\n1\nProbHit:\n0.95\nProbMiss:\n0.3\n"
           "FrameTransform:\n0.0 -1.0 0.0\n0.0 0.0 1.0\n1.0 0.0 0.0\n#endconfig\n")
    cfg = _write(tmp_path, "config.txt", "#config\nMappingRes:\n0.1\nProbHitThres:\n0.7\nProbMissThres:\n0.4\n"
                 "GridRes:\n0.1\nNodeEdge:\n8\nFrustumAllocationFactor:\n0.4\nFilterType:\n1\nUpdateType:\n0\n"
                 "PrecisionType:\n0\nPublishType:\n1\nUnknownKey:\nSensor:\ncam.txt\nSensor:\nvlp.txt\n#endconfig\n")
    h = load(cfg)
    i = info(h)
    assert i.filter_type == 1 and i.publish_sensor == 1
    assert i.clamp_min == np.float32(math.log(0.12) - math.log(0.88))
    assert i.clamp_max == np.float32(math.log(0.97) - math.log(0.03))
    _, d = sensor(h, 0)
    assert d.explicit_log_odds == 0 and d.hfov_deg == 0.0  # HFOV from the aspect ratio
    _, d = sensor(h, 1)
    assert (d.hres, d.vres) == (901, 16)
    md = N.NmMapDesc()
    N.call("nm_config_map_desc", h, C.byref(md))
    p = float(np.float32(0.7))  # the parsed float value of ProbHitThres
    assert md.thres_hit == np.float32(math.log(p) - math.log(1.0 - p))
    N.call("nm_config_destroy", h)


@pytest.mark.parametrize("text,needle", [
    ("#cfg\n#endconfig\n", b"expected #config"),
    ("#config\nMappingRes:\n0.1\n", b"missing #endconfig"),
    ("#config\nMappingRes:\nabc\n#endconfig\n", b"bad value"),
    ("#config\nSensor:\nnope.txt\n#endconfig\n", b"cannot open sensor config"),
    ("#config\nRounding:\nsideways\n#endconfig\n", b"Rounding"),
])
def test_malformed_configs_fail_with_io_errors(tmp_path, text, needle):
    cfg = _write(tmp_path, "bad.txt", text)
    h = C.c_void_p()
    rc = N.lib().nm_config_load(str(cfg).encode(), C.byref(h))
    assert rc == N.NM_ERR_IO and needle in N.lib().nm_last_error()


def test_missing_config_and_vdb_grid(tmp_path):
    h = C.c_void_p()
    assert N.lib().nm_config_load(str(tmp_path / "none.txt").encode(), C.byref(h)) == N.NM_ERR_IO


def test_facade_config_and_agent_accessors(tmp_path):
    """nanomap::config::Config's derived sizes (Config.cpp:24-58) and the Agent accessors of
    Agent.h:181-214 through the C++ facade, on the host only."""
    import subprocess
    root = Path(__file__).resolve().parents[1]
    exe = tmp_path / "config_demo"
    subprocess.run(["g++", "-std=c++17", "-O1", f"-I{root / 'include'}",
                    str(root / "tests" / "cpp" / "config_demo.cpp"), f"-L{root / 'nanomap_b200'}",
                    "-lnanomap_b200", f"-Wl,-rpath,{root / 'nanomap_b200'}", "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe), str(HEADLINE)], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    v = {}
    for line in out.stdout.splitlines():
        k, *rest = line.split()
        v[k] = rest
    assert v["leafVolume"] == ["512"]
    # the 640x480 camera and the 64x1024 spinning laser of the headline config
    assert v["maxPCLSize"] == ["307200"] and v["frustumPCLSize"] == ["307200"]
    assert v["laserPCLSize"] == ["65536"]
    # leaf box of the camera's 10 m range sphere at 0.05 m x 8: (ceil(20 / 0.4) + 2)^3
    assert v["frustumLeafBufferSize"] == [str(52 ** 3)]
    assert v["processType"] == ["1"] and v["laserVoxelBufferSize"] == ["0"]
    assert v["exploreType"] == ["0"] and v["simType"] == ["0"] and v["serialUpdate"] == ["0"]
    assert v["agentId"] == ["0"] and int(v["sensors"][0]) >= 1
    assert v["observationRays"] == ["80"] and v["observationNorms"] == ["80", "0.5", "20"]
    assert v["sensorsAfterReset"] == ["0"] and v["raysAfterReset"] == ["0"]
