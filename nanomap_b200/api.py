"""Python view of the C ABI, shaped like NanoMap's own objects (Pose, sensors, Map, sim map).

Used by the tests and the benchmark.  Arrays may be numpy arrays (host memory) or torch CUDA
tensors (device memory); the matching NM_INPUT_HOST / NM_OUTPUT_HOST flag is set from the
array type.  Every call goes through libnanomap_b200.so; nothing here computes a result.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N
from ._native import NanomapError, call, lib


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _ptr(x):
    """(pointer, is_host) of a numpy array or torch tensor."""
    if x is None:
        return None, True
    if _is_torch(x):
        if not x.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return C.c_void_p(x.data_ptr()), not x.is_cuda
    a = np.ascontiguousarray(x)
    if a is not x:
        raise ValueError("array must be C-contiguous")
    return C.c_void_p(a.ctypes.data), True


def _stream(stream):
    if stream is None:
        return None
    if isinstance(stream, int):
        return C.c_void_p(stream)
    return C.c_void_p(stream.cuda_stream)


def _ray_pose(position, rotation) -> N.NmRayPose:
    rp = N.NmRayPose()
    pos = np.asarray(position, np.float64).reshape(3)
    rot = np.asarray(rotation, np.float64).reshape(9)
    for i in range(3):
        rp.position[i] = float(pos[i])
    for i in range(9):
        rp.rotation[i] = float(rot[i])
    return rp


def observation_sphere(n: int) -> np.ndarray:
    """The n unit observation directions of an agent (Agent.h:147-192), (n, 3) float32."""
    out = np.zeros((n, 3), np.float32)
    call("nm_observation_sphere", n, out.ctypes.data_as(N._PF))
    return out


def make_pose(position, orientation) -> N.NmPose:
    p = N.NmPose()
    for i in range(3):
        p.position[i] = float(position[i])
    for i in range(4):
        p.orientation[i] = float(orientation[i])
    return p


@dataclass
class Pose:
    """nanomap::Pose: position (m) and quaternion (w, x, y, z); default (0,0,0,1) as in
    nanomap.h:24-25 (Eigen's (w, x, y, z) constructor order)."""
    position: tuple = (0.0, 0.0, 0.0)
    orientation: tuple = (0.0, 0.0, 0.0, 1.0)

    def c(self) -> N.NmPose:
        return make_pose(self.position, self.orientation)


def sensor_desc(type=0, hres=640, vres=480, hfov_deg=0.0, vfov_deg=58.0, min_range=0.0,
                max_range=10.0, prob_hit=0.7, prob_miss=0.4, log_odds_hit=0.0,
                log_odds_miss=0.0, explicit_log_odds=0, rate=30, frame_transform=None,
                id=0) -> N.NmSensorDesc:
    d = N.NmSensorDesc()
    d.type, d.id, d.hres, d.vres = type, id, hres, vres
    d.hfov_deg, d.vfov_deg = hfov_deg, vfov_deg
    d.min_range, d.max_range = min_range, max_range
    d.prob_hit, d.prob_miss = prob_hit, prob_miss
    d.log_odds_hit, d.log_odds_miss = log_odds_hit, log_odds_miss
    d.explicit_log_odds, d.rate = explicit_log_odds, rate
    ft = frame_transform if frame_transform is not None else (1, 0, 0, 0, 1, 0, 0, 0, 1)
    for i in range(9):
        d.frame_transform[i] = float(ft[i])
    return d


def map_desc(res=0.1, thres_hit=0.0, thres_miss=0.0, clamp_min=-2.0, clamp_max=3.5,
             clamp_mode=N.NM_CLAMP_ALWAYS, update_mode=N.NM_UPDATE_LABEL,
             rounding=N.NM_ROUND_DOWN, initial_leaf_capacity=0, max_agents=1) -> N.NmMapDesc:
    d = N.NmMapDesc()
    d.res, d.leaf_edge = res, 8
    d.thres_hit, d.thres_miss = thres_hit, thres_miss
    d.clamp_min, d.clamp_max = clamp_min, clamp_max
    d.clamp_mode, d.update_mode, d.rounding = clamp_mode, update_mode, rounding
    d.initial_leaf_capacity, d.max_agents = initial_leaf_capacity, max_agents
    return d


def frame_params(desc: N.NmSensorDesc, pose: Pose, res: float, rounding: int):
    """Host-only per-frame constants: (R[9], eye[3], max_time, pixel_model[6])."""
    R = (C.c_float * 9)()
    eye = (C.c_double * 3)()
    mt = C.c_float()
    pm = (C.c_float * 6)()
    call("nm_frame_params", C.byref(desc), C.byref(pose.c()), C.c_float(res), rounding, R, eye,
         C.byref(mt), pm)
    return (np.array(R[:], dtype=np.float32), np.array(eye[:], dtype=np.float64),
            np.float32(mt.value), np.array(pm[:], dtype=np.float32))


class Context:
    def __init__(self, device: int = 0):
        h = C.c_void_p()
        call("nm_context_create", device, C.byref(h))
        self.h = h
        self.device = device

    def sync(self):
        call("nm_context_sync", self.h)

    def close(self):
        if self.h:
            call("nm_context_destroy", self.h)
            self.h = None

    def add_noise(self, ranges, sigma_coef, drop_prob, seed, stream=None):
        p, host = _ptr(ranges)
        if host:
            raise ValueError("noise runs on device ranges")
        call("nm_ranges_add_noise", self.h, p, ranges.numel(), C.c_float(sigma_coef),
             C.c_float(drop_prob), C.c_uint64(seed), _stream(stream))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Sensor:
    def __init__(self, ctx: Context, desc: N.NmSensorDesc):
        self.ctx = ctx
        self.desc = desc
        h = C.c_void_p()
        call("nm_sensor_create", ctx.h, C.byref(desc), C.byref(h))
        self.h = h

    @property
    def shape(self):
        return (self.desc.vres, self.desc.hres)

    def params(self):
        out = (C.c_float * 6)()
        call("nm_sensor_params", self.h, out)
        return np.array(out[:], dtype=np.float32)

    def close(self):
        if self.h:
            call("nm_sensor_destroy", self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Map:
    """Device-resident occupancy map (replaces nanomap::map::Map + the handler's update)."""

    def __init__(self, ctx: Context, desc: N.NmMapDesc):
        self.ctx = ctx
        self.desc = desc
        h = C.c_void_p()
        call("nm_map_create", ctx.h, C.byref(desc), C.byref(h))
        self.h = h

    def insert_points(self, sensor: Sensor, pose: Pose, cloud, width: int, height: int,
                      step: int, flags: int = 0, stream=None):
        p, host = _ptr(cloud)
        if host:
            flags |= N.NM_INPUT_HOST
        call("nm_map_insert_points", self.h, sensor.h, C.byref(pose.c()), p, width, height,
             step, flags, _stream(stream))

    def insert_ranges(self, sensor: Sensor, pose: Pose, ranges, flags: int = 0, stream=None):
        p, host = _ptr(ranges)
        if host:
            flags |= N.NM_INPUT_HOST
        call("nm_map_insert_ranges", self.h, sensor.h, C.byref(pose.c()), p, flags,
             _stream(stream))

    def filter_points(self, sensor: Sensor, pose: Pose, data, width: int = 0, height: int = 0,
                      step: int = 0, centre: bool = False):
        """Voxel filter alone: (points (n,3) float32 world offsets from the sensor position,
        counts (n,) uint32) in voxel order.  step == 0: `data` is a range image of `sensor`."""
        p, host = _ptr(data)
        flags = N.NM_INPUT_HOST if host else 0
        if centre:
            flags |= N.NM_FILTER_CENTRE
        n = C.c_uint64()
        args = (self.h, sensor.h, C.byref(pose.c()), p, width, height, step)
        call("nm_map_filter_points", *args, flags, None, None, 0, C.byref(n))
        k = n.value
        pts = np.zeros((k, 3), np.float32)
        cnt = np.zeros(k, np.uint32)
        call("nm_map_filter_points", *args, flags, pts.ctypes.data_as(N._PF),
             cnt.ctypes.data_as(N._PU32), k, C.byref(n))
        return pts, cnt

    # ---- expected-depth rendering (device map read in place) ----------------------------
    @staticmethod
    def ray_pose(sensor: Sensor, pose: Pose):
        """(position (3,), rotation (3, 3)) float64 of the sensor, frame transform included."""
        rp = N.NmRayPose()
        call("nm_ray_pose_from_pose", sensor.h, C.byref(pose.c()), C.byref(rp))
        return np.array(rp.position[:]), np.array(rp.rotation[:]).reshape(3, 3)

    def values_copy(self):
        """The map's log-odds in slot layout as a (capacity, 512) float32 CUDA tensor."""
        import torch
        n = C.c_uint64()
        call("nm_map_values_copy", self.h, None, 0, C.byref(n), None)
        out = torch.empty(n.value, dtype=torch.float32, device="cuda")
        call("nm_map_values_copy", self.h, C.c_void_p(out.data_ptr()), n.value, C.byref(n),
             _stream(torch.cuda.current_stream()))
        return out.view(-1, 512)

    def slot_origins(self):
        """(capacity, 3) int32 leaf origin of every slot (INT32_MIN for empty slots)."""
        n = C.c_uint64()
        call("nm_map_slot_origins", self.h, None, 0, C.byref(n))
        out = np.zeros((n.value, 3), np.int32)
        call("nm_map_slot_origins", self.h, out.ctypes.data_as(N._PI32), n.value, C.byref(n))
        return out

    def depth_render(self, sensor: Sensor, position, rotation, values=None, scale=1.0,
                     bias=0.0):
        """Expected depth (vres, hres) float32 CUDA tensor at a float64 sensor pose."""
        import torch
        rp = _ray_pose(position, rotation)
        out = torch.empty((sensor.desc.vres, sensor.desc.hres), dtype=torch.float32, device="cuda")
        vp = C.c_void_p(values.data_ptr()) if values is not None else None
        nv = values.numel() if values is not None else 0
        call("nm_depth_render", self.h, sensor.h, C.byref(rp), vp, nv, scale, bias,
             C.c_void_p(out.data_ptr()), _stream(torch.cuda.current_stream()))
        return out

    def depth_backward(self, sensor: Sensor, position, rotation, grad_depth, values=None,
                       grad_values=None, scale=1.0, bias=0.0, depth=None):
        """Adds sum grad_depth * dD/dlog-odds into grad_values (slot layout) and returns
        sum grad_depth * dD/dxi (6,) float64 for xi = (rho, phi).  `depth`: depth_render's
        output for the same pose, values, scale and bias (one traversal replay fewer)."""
        import torch
        rp = _ray_pose(position, rotation)
        g = np.zeros(6)
        gd = grad_depth.contiguous()
        vp = C.c_void_p(values.data_ptr()) if values is not None else None
        gv = C.c_void_p(grad_values.data_ptr()) if grad_values is not None else None
        sizes = [t.numel() for t in (values, grad_values) if t is not None]
        nv = min(sizes) if sizes else 0
        dp = C.c_void_p(depth.contiguous().data_ptr()) if depth is not None else None
        call("nm_depth_backward", self.h, sensor.h, C.byref(rp), vp, nv, scale, bias,
             C.c_void_p(gd.data_ptr()), dp, gv, g.ctypes.data_as(N._PD),
             _stream(torch.cuda.current_stream()))
        return g

    def pose_refine(self, sensor: Sensor, position, rotation, target, steps=50,
                    lr_position=0.005, lr_rotation=0.002, scale=1.0, bias=0.0,
                    max_residual=0.0, surface_offset=0.0, edge_threshold=0.0):
        """Native Adam refinement (nm_pose_refine_desc); returns (position, rotation,
        losses (steps + 1,))."""
        import torch
        torch.cuda.current_stream().synchronize()
        rp = _ray_pose(position, rotation)
        losses = np.zeros(steps + 1, np.float32)
        t = target.contiguous()
        d = N.NmRefineDesc(scale, bias, max_residual, steps, lr_position, lr_rotation,
                           surface_offset, edge_threshold)
        call("nm_pose_refine_desc", self.h, sensor.h, C.byref(rp), C.c_void_p(t.data_ptr()),
             C.byref(d), losses.ctypes.data_as(N._PF))
        return np.array(rp.position[:]), np.array(rp.rotation[:]).reshape(3, 3), losses

    def set_launch(self, tile_w: int, tile_h: int, leaf_table_entries: int):
        call("nm_map_set_launch", self.h, tile_w, tile_h, leaf_table_entries)

    def integrate(self, stream=None):
        call("nm_map_integrate", self.h, _stream(stream))

    def tick(self, frames, flags: int = 0, stream=None):
        """frames: list of (sensor, pose, device ranges tensor, agent)."""
        arr = (N.NmFrame * len(frames))()
        for i, (s, pose, r, agent) in enumerate(frames):
            arr[i].sensor = s.h
            arr[i].pose = pose.c()
            arr[i].ranges = C.c_void_p(r.data_ptr())
            arr[i].agent = agent
        call("nm_map_tick", self.h, arr, len(frames), flags, _stream(stream))

    def status_async(self, out, stream=None):
        """Enqueue a copy of (leaf count, error bits) into `out` (2 x int32, page-locked host
        tensor), valid once the stream has passed this point."""
        p, host = _ptr(out)
        if not host:
            raise ValueError("status buffer must be host memory")
        call("nm_map_status_async", self.h, p, _stream(stream))

    def stats(self) -> dict:
        s = N.NmStats()
        call("nm_map_stats", self.h, C.byref(s))
        return {k: getattr(s, k) for k, _ in N.NmStats._fields_}

    def export(self):
        """(origins (n,3) int32, values (n,512) float32, active (n,16) uint32), any order."""
        n = C.c_uint64()
        call("nm_map_export", self.h, None, None, None, 0, C.byref(n))
        k = n.value
        o = np.zeros((k, 3), np.int32)
        v = np.zeros((k, 512), np.float32)
        a = np.zeros((k, 16), np.uint32)
        if k:
            call("nm_map_export", self.h, o.ctypes.data_as(N._PI32), v.ctypes.data_as(N._PF),
                 a.ctypes.data_as(N._PU32), k, C.byref(n))
        return o, v, a

    def export_labels(self, agent: int = 0):
        """(origins (n,3), words (n,32)) of leaves holding labels of one plane."""
        st = self.stats()
        cap = max(1, int(st["leaf_count"]))
        o = np.zeros((cap, 3), np.int32)
        w = np.zeros((cap, 32), np.uint32)
        n = C.c_uint64()
        call("nm_map_export_labels", self.h, agent, o.ctypes.data_as(N._PI32),
             w.ctypes.data_as(N._PU32), cap, C.byref(n))
        k = int(n.value)
        return o[:k].copy(), w[:k].copy()

    def frame_params(self, sensor: Sensor, pose: Pose):
        R = (C.c_float * 9)()
        eye = (C.c_double * 3)()
        mt = C.c_float()
        call("nm_map_frame_params", self.h, sensor.h, C.byref(pose.c()), R, eye, C.byref(mt))
        return np.array(R[:], np.float32), np.array(eye[:], np.float64), np.float32(mt.value)

    def reset(self):
        call("nm_map_reset", self.h)

    def close(self):
        if self.h:
            call("nm_map_destroy", self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class TickPlan:
    """A batched tick over fixed slots, replayed as a CUDA graph (nm_tick_plan_*)."""

    def __init__(self, m: "Map", slots, sim: "SimMap | None" = None):
        """slots: list of (sensor, device range tensor, agent plane)."""
        self.map = m
        self.slots = slots
        arr = (N.NmFrame * len(slots))()
        for i, (s, r, agent) in enumerate(slots):
            arr[i].sensor = s.h
            arr[i].ranges = C.c_void_p(r.data_ptr())
            arr[i].agent = agent
            arr[i].pose.orientation[0] = 1.0
        h = C.c_void_p()
        call("nm_tick_plan_create", m.h, sim.h if sim is not None else None, arr, len(slots), C.byref(h))
        self.h = h

    def set_pose(self, slot: int, pose: Pose):
        call("nm_tick_plan_set_pose", self.h, slot, C.byref(pose.c()))

    def set_noise(self, sigma_coef: float, drop_prob: float, seed: int):
        call("nm_tick_plan_set_noise", self.h, C.c_float(sigma_coef), C.c_float(drop_prob), C.c_uint64(seed))

    def set_launch(self, tile_w: int, tile_h: int, entries: int):
        call("nm_tick_plan_set_launch", self.h, tile_w, tile_h, entries)

    def run(self, flags: int = 0, stream=None):
        call("nm_tick_plan_run", self.h, flags, _stream(stream))

    def autotune(self, cache_path: str | None = None):
        best = (C.c_int32 * 3)()
        us = C.c_float()
        call("nm_tick_plan_autotune", self.h, cache_path.encode() if cache_path else None, best, C.byref(us))
        return tuple(best[:]), us.value

    def close(self):
        if self.h:
            call("nm_tick_plan_destroy", self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def vdb_active_voxels(path: str, grid: str | None = None):
    """nm_vdb_active_voxels: (voxel size (3,), translation (3,), active voxels (n, 3) int32) of
    a grid in an OpenVDB .vdb file; host only."""
    vs = np.zeros(3)
    tr = np.zeros(3)
    n = C.c_int64()
    g = grid.encode() if grid is not None else None
    call("nm_vdb_active_voxels", str(path).encode(), g, vs.ctypes.data_as(N._PD),
         tr.ctypes.data_as(N._PD), None, 0, C.byref(n))
    ijk = np.zeros((max(n.value, 1), 3), np.int32)
    call("nm_vdb_active_voxels", str(path).encode(), g, vs.ctypes.data_as(N._PD),
         tr.ctypes.data_as(N._PD), ijk.ctypes.data_as(N._PI32), n.value, C.byref(n))
    return vs, tr, ijk[:n.value]


def vdb_write_active_voxels(path: str, voxels, voxel_size: float, grid: str | None = None):
    """nm_vdb_write_active_voxels: voxels ((n, 3) int) as a float grid of a .vdb file."""
    v = np.ascontiguousarray(voxels, dtype=np.int32).reshape(-1, 3)
    call("nm_vdb_write_active_voxels", str(path).encode(), grid.encode() if grid else None,
         C.c_double(voxel_size), v.ctypes.data_as(N._PI32), len(v))


class SimMap:
    """Device sim map (replaces the NanoVDB sim grid of SimHandler)."""

    def __init__(self, ctx: Context, res: float, *, boxes=None, cylinders=None, vox_min=None,
                 vox_max=None, voxels=None):
        self.ctx = ctx
        self.res = res
        h = C.c_void_p()
        if voxels is not None:
            v = np.ascontiguousarray(voxels, dtype=np.int32)
            call("nm_simmap_create_voxels", ctx.h, C.c_float(res), v.ctypes.data_as(N._PI32),
                 len(v), C.byref(h))
        else:
            b = np.ascontiguousarray(boxes if boxes is not None else np.zeros((0, 6)), np.float64)
            c = np.ascontiguousarray(cylinders if cylinders is not None else np.zeros((0, 5)), np.float64)
            lo = (C.c_int32 * 3)(*vox_min)
            hi = (C.c_int32 * 3)(*vox_max)
            call("nm_simmap_create_primitives", ctx.h, C.c_float(res), lo, hi,
                 b.ctypes.data_as(N._PD), len(b), c.ctypes.data_as(N._PD), len(c), C.byref(h))
        self.h = h

    @classmethod
    def load(cls, ctx: Context, path: str) -> "SimMap":
        """nm_simmap_load: an OpenVDB .vdb grid or an NMSIMv1 voxel list."""
        h = C.c_void_p()
        call("nm_simmap_load", ctx.h, str(path).encode(), C.byref(h))
        return cls._adopt(ctx, None, h)

    def info(self):
        bb = (C.c_int32 * 6)()
        nv = C.c_uint64()
        nl = C.c_uint64()
        call("nm_simmap_info", self.h, bb, C.byref(nv), C.byref(nl))
        return tuple(bb[:]), nv.value, nl.value

    def export(self):
        _, _, nl = self.info()
        o = np.zeros((max(nl, 1), 3), np.int32)
        w = np.zeros((max(nl, 1), 16), np.uint32)
        n = C.c_uint64()
        call("nm_simmap_export", self.h, o.ctypes.data_as(N._PI32), w.ctypes.data_as(N._PU32),
             nl, C.byref(n))
        return o[:nl], w[:nl]

    def render(self, sensor: Sensor, pose: Pose, out, flags: int = 0, stream=None):
        p, host = _ptr(out)
        if host:
            flags |= N.NM_OUTPUT_HOST
        call("nm_sim_render", self.h, sensor.h, C.byref(pose.c()), p, flags, _stream(stream))

    def render_noisy(self, sensor: Sensor, pose: Pose, out, sigma_coef: float, drop: float,
                     seed: int, flags: int = 0, stream=None):
        """render() with the range noise of Context.add_noise applied in the same launch."""
        p, host = _ptr(out)
        if host:
            flags |= N.NM_OUTPUT_HOST
        call("nm_sim_render_noisy", self.h, sensor.h, C.byref(pose.c()), p, sigma_coef, drop,
             C.c_uint64(seed), flags, _stream(stream))

    def insert(self, m: "Map", sensor: Sensor, pose: Pose, sigma_coef: float = 0.0,
               drop: float = 0.0, seed: int = 0, out=None, flags: int = 0, stream=None):
        """Render this sensor's noisy range image and insert it into `m` (one launch in label
        mode); `out` (optional) receives the image."""
        p = None
        if out is not None:
            p, host = _ptr(out)
            if host:
                flags |= N.NM_OUTPUT_HOST
        call("nm_sim_insert", self.h, m.h, sensor.h, C.byref(pose.c()), sigma_coef, drop,
             C.c_uint64(seed), p, flags, _stream(stream))

    def cast_rays(self, origins, directions, max_range: float, stream=None):
        """Distances (metres) to the first active voxel along each ray within max_range, 0 when
        none.  numpy inputs give a numpy result; CUDA tensors give a CUDA tensor."""
        if _is_torch(origins):
            import torch
            o = origins.contiguous().float()
            d = directions.contiguous().float()
            out = torch.empty(o.numel() // 3, dtype=torch.float32, device=o.device)
            call("nm_sim_cast_rays", self.h, C.c_void_p(o.data_ptr()), C.c_void_p(d.data_ptr()),
                 out.numel(), max_range, C.c_void_p(out.data_ptr()), 0, _stream(stream))
            return out
        o = np.ascontiguousarray(origins, np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(directions, np.float32).reshape(-1, 3)
        out = np.zeros(len(o), np.float32)
        call("nm_sim_cast_rays", self.h, o.ctypes.data, d.ctypes.data, len(o), max_range,
             out.ctypes.data, N.NM_INPUT_HOST | N.NM_OUTPUT_HOST, _stream(stream))
        return out

    @classmethod
    def _adopt(cls, ctx: Context, res: float, handle: C.c_void_p) -> "SimMap":
        sm = cls.__new__(cls)
        sm.ctx = ctx
        sm.res = res
        sm.h = handle
        return sm

    def close(self):
        if self.h:
            call("nm_simmap_destroy", self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def cave_desc(map_size=(50.0, 50.0, 3.5), grid_res=0.1, fill_percentage=56, smoothing_count=4,
              active_max=4, active_min=4, seed=1, file_out="") -> N.NmCaveDesc:
    """A cave-generator description (the keys of a #cavegenconfig file); `seed` is the value
    srand receives."""
    d = N.NmCaveDesc()
    for a in range(3):
        d.map_size[a] = map_size[a]
    d.grid_res = grid_res
    d.fill_percentage = fill_percentage
    d.smoothing_count = smoothing_count
    d.active_max = active_max
    d.active_min = active_min
    d.seed = seed & 0xFFFFFFFF
    d.file_out = file_out.encode()
    return d


def load_cave_config(path) -> N.NmCaveDesc:
    d = N.NmCaveDesc()
    call("nm_cave_config_load", str(path).encode(), C.byref(d))
    return d


class Cave:
    """Procedural cave generator on the device (nanomap::mapgen::CaveGen)."""

    def __init__(self, ctx: Context, desc: N.NmCaveDesc):
        self.ctx = ctx
        self.desc = desc
        h = C.c_void_p()
        call("nm_cave_create", ctx.h, C.byref(desc), C.byref(h))
        self.h = h

    def dims(self):
        half = (C.c_int32 * 3)()
        cells = (C.c_int32 * 3)()
        call("nm_cave_dims", self.h, half, cells)
        return tuple(half[:]), tuple(cells[:])

    def populate(self, mode_2d=False, counter_rng=False):
        call("nm_cave_populate", self.h, (N.NM_CAVE_2D if mode_2d else 0) |
             (N.NM_CAVE_COUNTER_RNG if counter_rng else 0))

    def smooth(self, mode_2d=False):
        call("nm_cave_smooth", self.h, N.NM_CAVE_2D if mode_2d else 0)

    def floor_ceil(self):
        call("nm_cave_floor_ceil", self.h)

    def regions(self):
        n, big = C.c_int64(), C.c_int64()
        call("nm_cave_regions", self.h, C.byref(n), C.byref(big))
        return n.value, big.value

    def keep_largest(self):
        call("nm_cave_keep_largest", self.h)

    def cells(self) -> np.ndarray:
        n = C.c_int64()
        call("nm_cave_cells", self.h, None, 0, C.byref(n))
        out = np.zeros((max(n.value, 1), 3), np.int32)
        call("nm_cave_cells", self.h, out.ctypes.data_as(N._PI32), n.value, C.byref(n))
        return out[:n.value]

    def simmap(self, shell=True, half_width=3, closing=1) -> SimMap:
        h = C.c_void_p()
        call("nm_cave_simmap", self.h, int(shell), half_width, closing, C.byref(h))
        return SimMap._adopt(self.ctx, self.desc.grid_res, h)

    def save(self, path, shell=True, half_width=3, closing=1) -> str:
        written = C.create_string_buffer(512)
        call("nm_cave_save", self.h, int(shell), half_width, closing, str(path).encode(), written)
        return written.value.decode()

    def close(self):
        if self.h:
            call("nm_cave_destroy", self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def simmap_voxels(sm: SimMap) -> np.ndarray:
    """Active voxels of a sim map, sorted by (x, y, z)."""
    o, w = sm.export()
    if len(o) == 0:
        return np.zeros((0, 3), np.int32)
    bits = np.unpackbits(w.view(np.uint8).reshape(len(o), 64), axis=1, bitorder="little")
    leaf, l = np.nonzero(bits)
    v = np.stack([o[leaf, 0] + (l >> 6), o[leaf, 1] + ((l >> 3) & 7), o[leaf, 2] + (l & 7)], 1)
    idx = np.lexsort((v[:, 2], v[:, 1], v[:, 0]))
    return v[idx].astype(np.int32)


__all__ = ["Pose", "Context", "Sensor", "Map", "SimMap", "Cave", "cave_desc",
           "load_cave_config", "simmap_voxels", "sensor_desc", "map_desc", "frame_params",
           "NanomapError", "lib"]
