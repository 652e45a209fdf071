"""Seeded synthetic scenes and trajectories for the mapping and simulation workloads.

The reference evaluates on scenes it does not ship (procedural caves, ROS bags); these seeded
generators stand in for them with the shapes, sizes and value ranges of each workload:

* ``plain_small``  -- 20 x 20 x 5 m, 200 axis-aligned boxes (edges 0.2-2 m), sim grid 0.1 m,
  320x240 camera, 87 x 58 deg, 5 m range, mapping at 0.1 m.
* ``sim_headline`` -- 40 x 40 x 10 m, 2000 boxes (edges 0.1-3 m) and 300 vertical cylinders
  (radius 0.05-0.5 m, height 1-10 m), sim grid and mapping at 0.05 m, 640x480 camera,
  87 x 58 deg, 10 m range, range noise sigma = 0.005 d^2, 2 % of pixels dropped.
* ``large_fine``   -- 80 x 80 x 20 m, 10000 boxes and 2000 cylinders, 0.02 m, 1280x720 at
  15 m.

All randomness comes from splitmix64 streams (Steele, Lea and Flood, 2014), so the same seed
gives the same scene on every machine.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, n: int) -> np.ndarray:
    """n consecutive splitmix64 outputs for `seed` (uint64)."""
    with np.errstate(over="ignore"):
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + np.arange(1, n + 1, dtype=np.uint64) * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def uniform(seed: int, n: int, lo=0.0, hi=1.0) -> np.ndarray:
    u = (splitmix64(seed, n) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return lo + (hi - lo) * u


# FrameTransform of the reference's depth-camera config (optical z forward -> body x,
# optical x -> body -y, optical y -> body z), column-major as the config files store it.
OPTICAL_TO_BODY = (0.0, -1.0, 0.0, 0.0, 0.0, 1.0, 1.0, 0.0, 0.0)


@dataclass
class SceneSpec:
    name: str
    size: tuple
    n_boxes: int
    box_edge: tuple
    n_cyl: int = 0
    cyl_radius: tuple = (0.05, 0.5)
    cyl_height: tuple = (1.0, 10.0)
    sim_res: float = 0.1
    map_res: float = 0.1
    width: int = 320
    height: int = 240
    hfov: float = 87.0
    vfov: float = 58.0
    max_range: float = 5.0
    min_range: float = 0.0
    frames: int = 10
    agent_z: float = 1.5
    noise_coef: float = 0.0   # sigma = noise_coef * d^2
    noise_sigma: float = 0.0  # constant sigma (metres)
    drop: float = 0.0
    log_odds_hit: float = 0.85
    log_odds_miss: float = -0.4
    clamp: tuple = (-2.0, 3.5)


SCENES = {
    "plain_small": SceneSpec("plain_small", (20.0, 20.0, 5.0), 200, (0.2, 2.0), sim_res=0.1,
                             map_res=0.1, width=320, height=240, max_range=5.0, frames=10,
                             agent_z=1.5, noise_sigma=0.01),
    "sim_headline": SceneSpec("sim_headline", (40.0, 40.0, 10.0), 2000, (0.1, 3.0), n_cyl=300,
                              sim_res=0.05, map_res=0.05, width=640, height=480, max_range=10.0,
                              frames=100, agent_z=2.0, noise_coef=0.005, drop=0.02),
    "large_fine": SceneSpec("large_fine", (80.0, 80.0, 20.0), 10000, (0.1, 3.0), n_cyl=2000,
                            sim_res=0.02, map_res=0.02, width=1280, height=720, max_range=15.0,
                            frames=500, agent_z=2.0, noise_coef=0.005, drop=0.02),
}


@dataclass
class Scene:
    spec: SceneSpec
    boxes: np.ndarray      # (n, 6) float64: min xyz, max xyz (m)
    cylinders: np.ndarray  # (n, 5) float64: cx, cy, r, z0, z1 (m)
    vox_min: tuple = field(default=(0, 0, 0))
    vox_max: tuple = field(default=(0, 0, 0))


def make_scene(spec: SceneSpec | str, seed: int = 1) -> Scene:
    if isinstance(spec, str):
        spec = SCENES[spec]
    sx, sy, sz = spec.size
    nb = spec.n_boxes
    c = np.stack([uniform(seed * 16 + 1, nb, 0, sx), uniform(seed * 16 + 2, nb, 0, sy),
                  uniform(seed * 16 + 3, nb, 0, sz)], axis=1)
    e = np.stack([uniform(seed * 16 + 4 + a, nb, *spec.box_edge) for a in range(3)], axis=1)
    boxes = np.concatenate([c - e / 2, c + e / 2], axis=1)
    nc = spec.n_cyl
    cyl = np.zeros((nc, 5))
    if nc:
        cyl[:, 0] = uniform(seed * 16 + 8, nc, 0, sx)
        cyl[:, 1] = uniform(seed * 16 + 9, nc, 0, sy)
        cyl[:, 2] = uniform(seed * 16 + 10, nc, *spec.cyl_radius)
        cyl[:, 3] = 0.0
        cyl[:, 4] = np.minimum(uniform(seed * 16 + 11, nc, *spec.cyl_height), sz)
    vmax = tuple(int(math.ceil(s / spec.sim_res)) for s in spec.size)
    return Scene(spec, boxes, cyl, (0, 0, 0), vmax)


def occupied(scene: Scene, p, clearance: float = 0.0) -> bool:
    """Whether point p (m) lies inside a primitive grown by `clearance`, or outside the world."""
    p = np.asarray(p, dtype=np.float64)
    lo = np.zeros(3) + clearance
    hi = np.asarray(scene.spec.size) - clearance
    if np.any(p < lo) or np.any(p > hi):
        return True
    b = scene.boxes
    if len(b) and np.any(np.all((b[:, :3] - clearance <= p) & (p <= b[:, 3:] + clearance), axis=1)):
        return True
    cy = scene.cylinders
    if len(cy):
        d2 = (cy[:, 0] - p[0]) ** 2 + (cy[:, 1] - p[1]) ** 2
        inside = (d2 <= (cy[:, 2] + clearance) ** 2) & (cy[:, 3] - clearance <= p[2]) & (p[2] <= cy[:, 4] + clearance)
        if np.any(inside):
            return True
    return False


def yaw_quaternion(yaw: float) -> tuple:
    """(w, x, y, z) of a rotation by `yaw` radians about +z."""
    return (math.cos(yaw / 2), 0.0, 0.0, math.sin(yaw / 2))


def trajectory(scene: Scene, n: int | None = None, seed: int = 7, step: float = 0.2,
               yaw_step_deg: float = 5.0, clearance: float = 0.3):
    """Seeded random walk through free space: each frame moves `step` metres along the
    heading after turning by +-yaw_step; a blocked move turns further and retries.
    Returns a list of (position(3), quaternion(w,x,y,z)) at fixed height."""
    spec = scene.spec
    n = spec.frames if n is None else n
    z = spec.agent_z
    u = uniform(seed, 200000)
    k = 0

    def nxt():
        nonlocal k
        k += 1
        return u[(k - 1) % len(u)]

    pos = None
    for _ in range(20000):
        cand = np.array([0.1 * spec.size[0] + 0.8 * spec.size[0] * nxt(),
                         0.1 * spec.size[1] + 0.8 * spec.size[1] * nxt(), z])
        if not occupied(scene, cand, clearance):
            pos = cand
            break
    if pos is None:
        raise RuntimeError("no free start position found")
    yaw = 2 * math.pi * nxt()
    out = []
    for _ in range(n):
        out.append((tuple(float(v) for v in pos), yaw_quaternion(yaw)))
        turn = math.radians(yaw_step_deg) * (1 if nxt() < 0.5 else -1)
        moved = False
        for attempt in range(72):
            y2 = yaw + turn * (1 + attempt)
            cand = pos + step * np.array([math.cos(y2), math.sin(y2), 0.0])
            if not occupied(scene, cand, clearance):
                pos, yaw, moved = cand, y2, True
                break
        if not moved:
            yaw += math.pi
    return out


def voxels_from_leaves(origins, words) -> np.ndarray:
    """Active voxel coordinates (n, 3) int32 from leaf origins and 16-word bit masks."""
    origins = np.asarray(origins, np.int64)
    bits = np.unpackbits(np.ascontiguousarray(words, dtype="<u4").view(np.uint8), bitorder="little")
    bits = bits.reshape(len(origins), 512)
    leaf, l = np.nonzero(bits)
    local = np.stack([l >> 6, (l >> 3) & 7, l & 7], axis=1)
    return (origins[leaf] + local).astype(np.int32)


def write_nmsim(path, res: float, voxels) -> None:
    """Write an NMSIMv1 voxel list (the sim-grid file format nm_simmap_load reads)."""
    v = np.ascontiguousarray(voxels, dtype="<i4").reshape(-1, 3)
    with open(path, "wb") as f:
        f.write(b"NMSIMv1\0")
        f.write(np.float32(res).tobytes())
        f.write(np.int64(len(v)).tobytes())
        f.write(v.tobytes())


def sensor_desc_kwargs(spec: SceneSpec) -> dict:
    """Sensor parameters of a scene's camera (explicit log-odds, optical frame)."""
    return dict(type=0, hres=spec.width, vres=spec.height, hfov_deg=spec.hfov, vfov_deg=spec.vfov,
                min_range=spec.min_range, max_range=spec.max_range,
                log_odds_hit=spec.log_odds_hit, log_odds_miss=spec.log_odds_miss,
                explicit_log_odds=1, frame_transform=OPTICAL_TO_BODY)


# The batched multi-agent tick: the plain_small world mapped at 0.05 m into one shared map by
# 16 agents of uneven sensors, as (type, hres, vres, hfov deg, vfov deg, max range m): six
# 320x240 cameras at 5 m, six 640x480 at 10 m, three 1280x720 at 8 m (87 x 58 deg) and one
# spinning 64-beam x 1024-column range sensor (360 x 30 deg) at 20 m.
TICK_RES = 0.05
TICK_AGENTS = ([(0, 320, 240, 87.0, 58.0, 5.0)] * 6 + [(0, 640, 480, 87.0, 58.0, 10.0)] * 6 +
               [(0, 1280, 720, 87.0, 58.0, 8.0)] * 3 + [(1, 1024, 64, 360.0, 30.0, 20.0)])


def tick_agent_desc_kwargs(agent: tuple) -> dict:
    """Sensor parameters of one agent of the batched tick (explicit log-odds +0.85 / -0.4)."""
    typ, w, h, hf, vf, rng = agent
    return dict(type=typ, hres=w, vres=h, hfov_deg=hf, vfov_deg=vf, max_range=rng,
                explicit_log_odds=1, log_odds_hit=0.85, log_odds_miss=-0.4,
                frame_transform=OPTICAL_TO_BODY)


def tick_sim_box(spec: SceneSpec, res: float = TICK_RES):
    """Voxel box [0, size / res) of the batched tick's sim map."""
    return (0, 0, 0), tuple(int(math.ceil(x / res)) for x in spec.size)


def analytic_box_ranges(scene: Scene, pixel_model, width: int, height: int, max_range: float,
                        pos, q) -> np.ndarray:
    """Radial ranges (float32, 0 = no return) of a frustum camera against the scene's boxes by
    exact FP64 ray-box intersection: pixel (w, h) looks along (w/W * 2hw - hw, h/H * 2hh - hh,
    1) in the sensor frame (`pixel_model` = hw, hh, 2hw, 2hh, 1/W, 1/H)."""
    hw, hh, c0, c1 = (float(v) for v in pixel_model[:4])
    u = np.arange(width, dtype=np.float64) / width
    v = np.arange(height, dtype=np.float64) / height
    d = np.stack(np.broadcast_arrays(u[None, :] * c0 - hw, v[:, None] * c1 - hh, 1.0), axis=-1)
    m = d.reshape(-1, 3) @ rotation_matrix(q).T
    m /= np.linalg.norm(m, axis=1, keepdims=True)
    p = np.asarray(pos, dtype=np.float64)
    best = np.full(len(m), np.inf)
    # boxes whose nearest point lies beyond max range cannot be hit
    near = np.linalg.norm(np.maximum(np.maximum(scene.boxes[:, :3] - p, p - scene.boxes[:, 3:]), 0.0),
                          axis=1) <= max_range
    boxes = scene.boxes[near]
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = 1.0 / m
        for c in range(0, len(boxes), 64):  # slab tests of 64 boxes at a time
            b = boxes[c:c + 64]
            t0 = np.zeros((len(m), len(b)))
            t1 = np.full((len(m), len(b)), np.inf)
            for a in range(3):  # fmax / fmin skip the NaN of 0 * inf on a parallel axis
                ta = (b[None, :, a] - p[a]) * inv[:, a, None]
                tb = (b[None, :, 3 + a] - p[a]) * inv[:, a, None]
                t0 = np.fmax(t0, np.fmin(ta, tb))
                t1 = np.fmin(t1, np.fmax(ta, tb))
            best = np.minimum(best, np.where(t0 <= t1, t0, np.inf).min(axis=1))
    out = np.where((best <= max_range) & (best > 0.0), best, 0.0)
    return out.astype(np.float32).reshape(height, width)


def rotation_matrix(q, F=OPTICAL_TO_BODY) -> np.ndarray:
    """World-from-sensor rotation in float64 (for analytic rendering; not bit-matched)."""
    w, x, y, z = q
    n = math.sqrt(w * w + x * x + y * y + z * z)
    w, x, y, z = w / n, x / n, y / n, z / n
    M = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                  [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                  [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])
    Fm = np.array(F, dtype=np.float64).reshape(3, 3).T  # column-major -> matrix
    return M @ Fm
