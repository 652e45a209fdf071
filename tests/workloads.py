"""Shared test workloads: seeded scenes, poses and range images, plus oracle helpers."""
from __future__ import annotations

import numpy as np

from nanomap_b200 import scenes as S
from nanomap_b200.api import Pose, sensor_desc
from nanomap_b200.diff import so3_exp
from oracle import oracle as O


def camera_desc(spec: S.SceneSpec, **over):
    kw = S.sensor_desc_kwargs(spec)
    kw.update(over)
    return sensor_desc(**kw)


def plain_small_frames(n=10, seed=1, noise=True):
    """The small plain-mapping workload: analytic FP64 box ranges + N(0, 0.01 m) noise."""
    spec = S.SCENES["plain_small"]
    scene = S.make_scene(spec, seed)
    traj = S.trajectory(scene, n, seed=seed + 6)
    desc = camera_desc(spec)
    osen = O.Sensor.from_desc(desc)
    rng = np.random.default_rng(seed + 100)
    frames = []
    for pos, q in traj:
        R64 = S.rotation_matrix(q)
        r = O.render_boxes(osen, pos, R64, scene.boxes)
        if noise:
            valid = r > 0
            r = np.where(valid, r + rng.normal(0.0, spec.noise_sigma, r.shape), 0.0).astype(np.float32)
            r[~(r > 0)] = 0.0
        frames.append((Pose(pos, q), r.astype(np.float32)))
    return spec, scene, desc, frames


def oracle_frame(desc, pose: Pose, res: float, rounding: int):
    R = O.rotation(pose.orientation, list(desc.frame_transform))
    eye, mt = O.frame_setup(pose.position, res, desc.max_range, rounding)
    return R, eye, mt


def active_bits_from_bytes(active_u8: np.ndarray) -> np.ndarray:
    """(n, 512) bytes -> (n, 16) uint32 words, bit l%32 of word l/32 = voxel l."""
    a = active_u8.astype(np.uint32).reshape(-1, 16, 32)
    return (a << np.arange(32, dtype=np.uint32)).sum(axis=2).astype(np.uint32)


def leaf_dict(origins, *arrays):
    return {tuple(int(v) for v in o): tuple(a[i] for a in arrays) for i, o in enumerate(origins)}


def compare_maps(gpu_export, other_export):
    """Mismatch descriptions between a GPU export and another export (an oracle export with
    512 active bytes per leaf, or a second GPU export with 16 active words per leaf)."""
    go, gv, ga = gpu_export
    oo, ov, oa = other_export
    G = leaf_dict(go, gv, ga)
    Od = leaf_dict(oo, ov, oa if oa.shape[1:] == (16,) else active_bits_from_bytes(oa))
    errs = []
    zero_v = np.zeros(512, np.float32)
    zero_a = np.zeros(16, np.uint32)
    for k in set(G) | set(Od):
        gv_, ga_ = G.get(k, (zero_v, zero_a))
        ov_, oa_ = Od.get(k, (zero_v, zero_a))
        if not np.array_equal(gv_.view(np.uint32), ov_.view(np.uint32)):
            d = np.nonzero(gv_.view(np.uint32) != ov_.view(np.uint32))[0]
            errs.append(f"leaf {k}: {len(d)} values differ, e.g. voxel {d[0]}: {gv_[d[0]]!r} vs {ov_[d[0]]!r}")
        if not np.array_equal(ga_, oa_):
            errs.append(f"leaf {k}: active bits differ")
        if len(errs) > 20:
            break
    return errs


def compare_labels(gpu_labels, oracle_labels):
    go, gw = gpu_labels
    oo, ow = oracle_labels
    G = leaf_dict(go, gw)
    Od = leaf_dict(oo, ow)
    errs = []
    for k in set(G) | set(Od):
        a = G.get(k, (np.zeros(32, np.uint32),))[0]
        b = Od.get(k, (np.zeros(32, np.uint32),))[0]
        if not np.array_equal(a, b):
            errs.append(f"leaf {k}: labels differ in words {np.nonzero(a != b)[0].tolist()}")
        if len(errs) > 20:
            break
    return errs


def central_differences(render, pos, R, h, n):
    """FP64 central differences of render(pos, R) -> (values (n,), hashes) for the six pose
    components at step h, and the mask of (pixel, component) pairs whose voxel sequence is the
    same at both perturbed poses."""
    _, base_hash = render(pos, R)
    fd = np.zeros((n, 6))
    ok = np.ones((n, 6), bool)
    for i in range(6):
        for sgn in (1.0, -1.0):
            p2, R2 = pos.copy(), R
            if i < 3:
                p2[i] += sgn * h
            else:
                phi = np.zeros(3)
                phi[i - 3] = sgn * h
                R2 = so3_exp(phi) @ R
            D2, h2 = render(p2, R2)
            ok[:, i] &= h2 == base_hash
            fd[:, i] += sgn * D2 / (2 * h)
    return fd, ok


def richardson(render, pos, R, h, n):
    """Central differences at h and h/2 combined to cancel the h^2 error term."""
    f1, ok1 = central_differences(render, pos, R, h, n)
    f2, ok2 = central_differences(render, pos, R, h / 2, n)
    return (4.0 * f2 - f1) / 3.0, ok1 & ok2
