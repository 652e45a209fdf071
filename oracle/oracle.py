"""ctypes wrapper of the CPU oracle (oracle/nm_oracle.cpp) -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py (cpu_baseline and --impl reference) import
this module.  It is the checker, never the thing measured as the product.

PARITY UNPINNED: see the header of nm_oracle.cpp -- the reference has no golden vectors and
cannot be built here; the oracle is pinned by hand-derived known-answer cases only.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"

_PF = C.POINTER(C.c_float)
_PD = C.POINTER(C.c_double)
_PI32 = C.POINTER(C.c_int32)
_PU32 = C.POINTER(C.c_uint32)
_PU8 = C.POINTER(C.c_uint8)
_PI64 = C.POINTER(C.c_int64)


class OrcSensor(C.Structure):
    _fields_ = [
        ("type", C.c_int32), ("width", C.c_int32), ("height", C.c_int32), ("pad", C.c_int32),
        ("hw", C.c_float), ("hh", C.c_float), ("c0", C.c_float), ("c1", C.c_float),
        ("scale_u", C.c_float), ("scale_v", C.c_float),
        ("min_range", C.c_float), ("max_range", C.c_float),
        ("sinu", _PF), ("cosu", _PF), ("sinv", _PF), ("cosv", _PF),
    ]


class OrcMapParams(C.Structure):
    _fields_ = [
        ("res", C.c_float), ("thres_hit", C.c_float), ("thres_miss", C.c_float),
        ("clamp_min", C.c_float), ("clamp_max", C.c_float),
        ("clamp_mode", C.c_int32), ("update_mode", C.c_int32), ("rounding", C.c_int32),
    ]


_lib = None


def build() -> Path:
    subprocess.run(["make", "-C", str(HERE), "-s"], check=True)
    return LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        L.orc_rotation.argtypes = [_PF, _PF, _PF]
        L.orc_frame_setup.argtypes = [_PF, C.c_float, C.c_float, C.c_int, _PD, _PF]
        L.orc_frustum_params.argtypes = [C.c_int, C.c_int, C.c_float, C.c_float, _PF]
        L.orc_laser_tables.argtypes = [C.c_int, C.c_int, C.c_float, C.c_float, _PF, _PF, _PF, _PF]
        L.orc_ranges_to_points.argtypes = [C.POINTER(OrcSensor), _PF, _PF]
        L.orc_trace.argtypes = [_PF, _PD, C.c_double, C.c_float, C.c_int, C.c_float, C.c_float,
                                C.c_float, _PI32, C.c_int64]
        L.orc_trace.restype = C.c_int64
        L.orc_map_create.argtypes = [C.POINTER(OrcMapParams)]
        L.orc_map_create.restype = C.c_void_p
        L.orc_map_destroy.argtypes = [C.c_void_p]
        L.orc_map_insert.argtypes = [C.c_void_p, _PF, _PD, C.c_double, C.c_float, C.c_float,
                                     C.c_float, _PF, C.c_int64, C.c_int64, C.c_int, C.c_int]
        L.orc_map_labels.argtypes = [C.c_void_p, _PI32, _PU32, C.c_int64]
        L.orc_map_labels.restype = C.c_int64
        L.orc_map_export.argtypes = [C.c_void_p, _PI32, _PF, _PU8, C.c_int64]
        L.orc_map_export.restype = C.c_int64
        L.orc_map_stats.argtypes = [C.c_void_p, _PI64]
        L.orc_simmap_create.argtypes = [C.c_float, _PI32, _PI32, _PD, C.c_int, _PD, C.c_int]
        L.orc_simmap_create.restype = C.c_void_p
        L.orc_simmap_from_voxels.argtypes = [C.c_float, _PI32, C.c_int64]
        L.orc_simmap_from_voxels.restype = C.c_void_p
        L.orc_simmap_destroy.argtypes = [C.c_void_p]
        L.orc_simmap_bbox.argtypes = [C.c_void_p, _PI32]
        L.orc_simmap_export.argtypes = [C.c_void_p, _PI32, _PU32, C.c_int64]
        L.orc_simmap_export.restype = C.c_int64
        L.orc_simmap_count.argtypes = [C.c_void_p]
        L.orc_simmap_count.restype = C.c_int64
        L.orc_sim_render.argtypes = [C.c_void_p, C.POINTER(OrcSensor), _PF, _PF, _PF, C.c_int]
        L.orc_voxel_filter.argtypes = [_PF, _PD, C.c_double, C.c_float, C.c_int, C.c_int, _PF, C.c_int64,
                                        C.c_int64, _PF, _PU32, C.c_int64]
        L.orc_voxel_filter.restype = C.c_int64
        L.orc_render_boxes.argtypes = [C.POINTER(OrcSensor), _PD, _PD, _PD, C.c_int, _PF]
        L.orc_sim_cast.argtypes = [C.c_void_p, _PF, _PF, C.c_int64, C.c_float, _PF]
        L.orc_depth_set_stop.argtypes = [C.c_double]
        L.orc_depth.argtypes = [C.POINTER(OrcSensor), _PD, _PD, C.c_double, _PI32, _PF, C.c_int64,
                                C.c_double, C.c_double, _PI32, C.c_int64, _PD, _PD,
                                C.POINTER(C.c_uint64), _PD, _PD]
        L.orc_cave_new.argtypes = [_PD, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint32]
        L.orc_cave_new.restype = C.c_void_p
        L.orc_cave_free.argtypes = [C.c_void_p]
        L.orc_cave_dims.argtypes = [C.c_void_p, _PI32]
        L.orc_cave_populate.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.orc_cave_smooth.argtypes = [C.c_void_p, C.c_int]
        L.orc_cave_floor_ceil.argtypes = [C.c_void_p]
        L.orc_cave_set_cells.argtypes = [C.c_void_p, _PI32, C.c_int64]
        L.orc_cave_regions.argtypes = [C.c_void_p, _PI64, _PI64]
        L.orc_cave_keep_largest.argtypes = [C.c_void_p]
        L.orc_cave_cells.argtypes = [C.c_void_p, _PI32, C.c_int64]
        L.orc_cave_cells.restype = C.c_int64
        L.orc_cave_voxels.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, _PI32, C.c_int64]
        L.orc_cave_voxels.restype = C.c_int64
        _lib = L
    return _lib


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def fp(a):
    return a.ctypes.data_as(_PF)


def dp(a):
    return a.ctypes.data_as(_PD)


def rotation(q, F) -> np.ndarray:
    R = np.zeros(9, np.float32)
    q = _f(q)
    F = _f(F)
    lib().orc_rotation(fp(q), fp(F), fp(R))
    return R


def frame_setup(pos, res, max_range, rounding):
    eye = np.zeros(3, np.float64)
    mt = C.c_float()
    p = _f(pos)
    lib().orc_frame_setup(fp(p), C.c_float(res), C.c_float(max_range), rounding, dp(eye), C.byref(mt))
    return eye, np.float32(mt.value)


class Sensor:
    """Oracle-side pixel model of a sensor (frustum or laser)."""

    def __init__(self, type=0, width=320, height=240, hfov_deg=0.0, vfov_deg=58.0,
                 min_range=0.0, max_range=5.0):
        self.s = OrcSensor()
        self.s.type, self.s.width, self.s.height = type, width, height
        self.s.min_range, self.s.max_range = min_range, max_range
        self.keep = []
        if type == 0:
            out = np.zeros(6, np.float32)
            lib().orc_frustum_params(width, height, C.c_float(hfov_deg), C.c_float(vfov_deg), fp(out))
            (self.s.hw, self.s.hh, self.s.c0, self.s.c1, self.s.scale_u, self.s.scale_v) = [float(x) for x in out]
            self.params = out
        else:
            su, cu = np.zeros(width, np.float32), np.zeros(width, np.float32)
            sv, cv = np.zeros(height, np.float32), np.zeros(height, np.float32)
            lib().orc_laser_tables(width, height, C.c_float(hfov_deg), C.c_float(vfov_deg),
                                   fp(su), fp(cu), fp(sv), fp(cv))
            self.keep = [su, cu, sv, cv]
            self.s.sinu, self.s.cosu, self.s.sinv, self.s.cosv = fp(su), fp(cu), fp(sv), fp(cv)
            self.params = np.zeros(6, np.float32)

    @classmethod
    def from_desc(cls, d):
        return cls(d.type, d.hres, d.vres, d.hfov_deg, d.vfov_deg, d.min_range, d.max_range)

    def points(self, ranges) -> np.ndarray:
        r = _f(ranges).reshape(-1)
        out = np.zeros((len(r), 3), np.float32)
        lib().orc_ranges_to_points(C.byref(self.s), fp(r), fp(out))
        return out


def trace(R, eye, res_d, max_time, rounding, p):
    R = _f(R)
    eye = _d(eye)
    buf = np.zeros((4096, 4), np.int32)
    n = lib().orc_trace(fp(R), dp(eye), C.c_double(res_d), C.c_float(max_time), rounding,
                        C.c_float(p[0]), C.c_float(p[1]), C.c_float(p[2]),
                        buf.ctypes.data_as(_PI32), 4096)
    if n > 4096:
        buf = np.zeros((n, 4), np.int32)
        lib().orc_trace(fp(R), dp(eye), C.c_double(res_d), C.c_float(max_time), rounding,
                        C.c_float(p[0]), C.c_float(p[1]), C.c_float(p[2]),
                        buf.ctypes.data_as(_PI32), n)
    return buf[: max(n, 0)].copy() if n >= 0 else None


class Map:
    """Oracle occupancy map (sparse leaves keyed by leaf coordinate)."""

    def __init__(self, res, clamp_min=-2.0, clamp_max=3.5, thres_hit=0.0, thres_miss=0.0,
                 clamp_mode=0, update_mode=0, rounding=1):
        p = OrcMapParams()
        p.res, p.thres_hit, p.thres_miss = res, thres_hit, thres_miss
        p.clamp_min, p.clamp_max = clamp_min, clamp_max
        p.clamp_mode, p.update_mode, p.rounding = clamp_mode, update_mode, rounding
        self.p = p
        self.h = lib().orc_map_create(C.byref(p))

    def insert(self, R, eye, max_time, lh, lm, points, threads=1, keep_labels=False):
        pts = _f(points).reshape(-1, 3)
        R = _f(R)
        eye = _d(eye)
        lib().orc_map_insert(self.h, fp(R), dp(eye), C.c_double(float(np.float32(self.p.res))),
                             C.c_float(max_time), C.c_float(lh), C.c_float(lm), fp(pts),
                             len(pts), 3, threads, 1 if keep_labels else 0)

    def insert_strided(self, R, eye, max_time, lh, lm, buf_f32, n, stride_floats, threads=1,
                       keep_labels=False):
        R = _f(R)
        eye = _d(eye)
        lib().orc_map_insert(self.h, fp(R), dp(eye), C.c_double(float(np.float32(self.p.res))),
                             C.c_float(max_time), C.c_float(lh), C.c_float(lm), fp(buf_f32), n,
                             stride_floats, threads, 1 if keep_labels else 0)

    def labels(self):
        n = lib().orc_map_labels(self.h, None, None, 0)
        o = np.zeros((n, 3), np.int32)
        w = np.zeros((n, 32), np.uint32)
        if n:
            lib().orc_map_labels(self.h, o.ctypes.data_as(_PI32), w.ctypes.data_as(_PU32), n)
        return o, w

    def export(self):
        n = lib().orc_map_export(self.h, None, None, None, 0)
        o = np.zeros((n, 3), np.int32)
        v = np.zeros((n, 512), np.float32)
        a = np.zeros((n, 512), np.uint8)
        if n:
            lib().orc_map_export(self.h, o.ctypes.data_as(_PI32), fp(v), a.ctypes.data_as(_PU8), n)
        return o, v, a

    def stats(self):
        out = np.zeros(4, np.int64)
        lib().orc_map_stats(self.h, out.ctypes.data_as(_PI64))
        return dict(visits=int(out[0]), rays=int(out[1]), unique_voxels=int(out[2]), leaves=int(out[3]))

    def __del__(self):
        try:
            lib().orc_map_destroy(self.h)
        except Exception:
            pass


class SimMap:
    def __init__(self, res, vox_min=None, vox_max=None, boxes=None, cylinders=None, voxels=None):
        self.res = res
        if voxels is not None:
            v = np.ascontiguousarray(voxels, np.int32)
            self.h = lib().orc_simmap_from_voxels(C.c_float(res), v.ctypes.data_as(_PI32), len(v))
        else:
            b = _d(boxes if boxes is not None else np.zeros((0, 6)))
            c = _d(cylinders if cylinders is not None else np.zeros((0, 5)))
            lo = np.ascontiguousarray(vox_min, np.int32)
            hi = np.ascontiguousarray(vox_max, np.int32)
            self.h = lib().orc_simmap_create(C.c_float(res), lo.ctypes.data_as(_PI32),
                                             hi.ctypes.data_as(_PI32), dp(b), len(b), dp(c), len(c))

    def bbox(self):
        out = np.zeros(7, np.int32)
        lib().orc_simmap_bbox(self.h, out.ctypes.data_as(_PI32))
        return tuple(out[:6]), bool(out[6])

    def count(self):
        return int(lib().orc_simmap_count(self.h))

    def export(self):
        n = lib().orc_simmap_export(self.h, None, None, 0)
        o = np.zeros((n, 3), np.int32)
        w = np.zeros((n, 16), np.uint32)
        if n:
            lib().orc_simmap_export(self.h, o.ctypes.data_as(_PI32), w.ctypes.data_as(_PU32), n)
        return o, w

    def cast(self, origins, directions, max_range) -> np.ndarray:
        o = _f(origins).reshape(-1, 3)
        d = _f(directions).reshape(-1, 3)
        out = np.zeros(len(o), np.float32)
        lib().orc_sim_cast(self.h, fp(o), fp(d), len(o), C.c_float(max_range), fp(out))
        return out

    def render(self, sensor: Sensor, pos, R, threads: int = 1) -> np.ndarray:
        out = np.zeros((sensor.s.height, sensor.s.width), np.float32)
        p = _f(pos)
        R = _f(R)
        lib().orc_sim_render(self.h, C.byref(sensor.s), fp(p), fp(R), fp(out), threads)
        return out

    def __del__(self):
        try:
            lib().orc_simmap_destroy(self.h)
        except Exception:
            pass


def render_boxes(sensor: Sensor, pos, R64, boxes) -> np.ndarray:
    out = np.zeros((sensor.s.height, sensor.s.width), np.float32)
    p = _d(pos)
    R = _d(R64).reshape(-1)
    b = _d(boxes)
    lib().orc_render_boxes(C.byref(sensor.s), dp(p), dp(R), dp(b), len(b), fp(out))
    return out


def voxel_filter(R, eye, res, max_time, rounding, points, centre=False):
    """Filtered points (world offsets from the eye, metres) and counts, sorted by voxel key."""
    pts = _f(points).reshape(-1, 3)
    R = _f(R)
    eye = _d(eye)
    args = (fp(R), dp(eye), C.c_double(float(np.float32(res))), C.c_float(max_time), rounding,
            1 if centre else 0, fp(pts), len(pts), 3)
    n = lib().orc_voxel_filter(*args, None, None, 0)
    out = np.zeros((n, 3), np.float32)
    cnt = np.zeros(n, np.uint32)
    lib().orc_voxel_filter(*args, fp(out), cnt.ctypes.data_as(_PU32), n)
    return out, cnt


def depth(sensor: Sensor, pos, R, res, origins, values, scale=1.0, bias=0.0, pixels=None,
          grad_depth=None, want_grad=True, stop_transmittance=0.0):
    """FP64 expected depth of the listed pixels (all when None) over a map given as leaf
    origins (n, 3) and values (n, 512).  Returns (depth (m), dpose (n_pix, 6): d/drho, d/dphi,
    sequence hashes, grad_values (n, 512) of sum grad_depth * depth or None).
    stop_transmittance > 0 leaves out each ray's voxels after its transmittance falls below
    it (the definition walks to max range)."""
    s = sensor.s
    if pixels is None:
        pixels = np.arange(s.width * s.height, dtype=np.int32)
    pixels = np.ascontiguousarray(pixels, np.int32)
    origins = np.ascontiguousarray(origins, np.int32).reshape(-1, 3)
    values = _f(values).reshape(-1, 512)
    n = len(pixels)
    out = np.zeros(n)
    dpose = np.zeros((n, 6)) if want_grad else None
    hashes = np.zeros(n, np.uint64)
    gv = None
    gd = None
    if grad_depth is not None:
        gd = _d(grad_depth).reshape(-1)
        gv = np.zeros((len(origins), 512))
    lib().orc_depth_set_stop(C.c_double(stop_transmittance))
    lib().orc_depth(C.byref(s), dp(_d(pos)), dp(_d(R).reshape(-1)), C.c_double(res),
                    origins.ctypes.data_as(_PI32), fp(values), len(origins), C.c_double(scale),
                    C.c_double(bias), pixels.ctypes.data_as(_PI32), n, dp(out),
                    dp(dpose) if dpose is not None else None,
                    hashes.ctypes.data_as(C.POINTER(C.c_uint64)),
                    dp(gd) if gd is not None else None, dp(gv) if gv is not None else None)
    return out, dpose, hashes, gv


def sort_leaves(origins, *arrays):
    """Sort leaf arrays by origin (x, y, z) so two exports can be compared row by row."""
    if len(origins) == 0:
        return (origins,) + arrays
    idx = np.lexsort((origins[:, 2], origins[:, 1], origins[:, 0]))
    return (origins[idx],) + tuple(a[idx] for a in arrays)


class Cave:
    """CaveGen restated on a sparse coordinate set (oracle/nm_oracle_cave.cpp)."""

    def __init__(self, map_size, grid_res, fill_percentage, smoothing_count, active_max,
                 active_min, seed):
        size = np.ascontiguousarray(map_size, np.float64)
        self.h = lib().orc_cave_new(dp(size), C.c_double(grid_res), int(fill_percentage),
                                    int(smoothing_count), int(active_max), int(active_min),
                                    C.c_uint32(int(seed) & 0xFFFFFFFF))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_cave_free(self.h)
            self.h = None

    def dims(self):
        d = np.zeros(3, np.int32)
        lib().orc_cave_dims(self.h, d.ctypes.data_as(_PI32))
        return tuple(int(v) for v in d)

    def populate(self, mode_2d=False, counter=False):
        lib().orc_cave_populate(self.h, int(mode_2d), int(counter))

    def smooth(self, mode_2d=False):
        lib().orc_cave_smooth(self.h, int(mode_2d))

    def floor_ceil(self):
        lib().orc_cave_floor_ceil(self.h)

    def set_cells(self, xyz):
        v = np.ascontiguousarray(xyz, np.int32).reshape(-1, 3)
        lib().orc_cave_set_cells(self.h, v.ctypes.data_as(_PI32), len(v))

    def regions(self):
        n, big = C.c_int64(0), C.c_int64(0)
        lib().orc_cave_regions(self.h, C.byref(n), C.byref(big))
        return n.value, big.value

    def keep_largest(self):
        lib().orc_cave_keep_largest(self.h)

    def cells(self) -> np.ndarray:
        n = lib().orc_cave_cells(self.h, None, 0)
        out = np.zeros((max(n, 1), 3), np.int32)
        lib().orc_cave_cells(self.h, out.ctypes.data_as(_PI32), n)
        return out[:n]

    def voxels(self, shell=True, half_width=3, closing=1) -> np.ndarray:
        n = lib().orc_cave_voxels(self.h, int(shell), half_width, closing, None, 0)
        out = np.zeros((max(n, 1), 3), np.int32)
        lib().orc_cave_voxels(self.h, int(shell), half_width, closing, out.ctypes.data_as(_PI32), n)
        return out[:n]
