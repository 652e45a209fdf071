"""The FP64 expected-depth definition (oracle) against its own central finite differences.

The oracle's analytic gradients (log-odds and se(3) pose) are what the GPU adjoint is checked
against, so they are pinned here to FP64 central differences first.  A pixel takes part in a
pose component only when its voxel sequence (while the transmittance is above 1e-12) is the
same at both perturbed poses: across such a change the expected depth has a kink and a
central difference does not estimate the derivative.
"""
import numpy as np

from nanomap_b200 import scenes as S
from nanomap_b200.diff import so3_exp
from oracle import oracle as O
from tests.workloads import oracle_frame, plain_small_frames, richardson


def _small_map():
    spec, scene, desc, frames = plain_small_frames(n=6)
    res = spec.map_res
    om = O.Map(res, clamp_min=spec.clamp[0], clamp_max=spec.clamp[1], rounding=1)
    osen = O.Sensor.from_desc(desc)
    for pose, ranges in frames:
        R, eye, mt = oracle_frame(desc, pose, res, 1)
        om.insert(R, eye, mt, desc.log_odds_hit, desc.log_odds_miss, osen.points(ranges))
    org, val, _ = om.export()
    return spec, desc, frames, osen, float(np.float32(res)), org, val


def _perturbed(frames, seed=3):
    rng = np.random.default_rng(seed)
    pose = frames[3][0]
    pos = np.array(pose.position, float) + rng.uniform(-0.05, 0.05, 3)
    R = so3_exp(np.radians(rng.uniform(-2, 2, 3))) @ S.rotation_matrix(pose.orientation)
    return pos, R


def test_pose_gradient_matches_central_differences():
    spec, desc, frames, osen, res, org, val = _small_map()
    pos, R = _perturbed(frames)
    pix = np.random.default_rng(7).choice(desc.hres * desc.vres, 64, replace=False).astype(np.int32)
    for scale, bias in ((1.0, 0.0), (3.0, -1.0)):
        D, dpose, hs, _ = O.depth(osen, pos, R, res, org, val, scale=scale, bias=bias, pixels=pix)

        def render(p2, R2):
            D2, _, h2, _ = O.depth(osen, p2, R2, res, org, val, scale=scale, bias=bias,
                                   pixels=pix, want_grad=False)
            return D2, h2

        fd, ok = richardson(render, pos, R, 1e-4, 64)
        assert ok.sum(axis=0).min() >= 40, ok.sum(axis=0)
        g = (dpose * ok).sum(axis=0)
        f = (fd * ok).sum(axis=0)
        for blk in (slice(0, 3), slice(3, 6)):
            assert np.abs(g[blk] - f[blk]).max() <= 1e-6 * np.abs(f[blk]).max(), (scale, g, f)


def test_logodds_gradient_matches_central_differences():
    spec, desc, frames, osen, res, org, val = _small_map()
    pos, R = _perturbed(frames)
    pix = np.random.default_rng(8).choice(desc.hres * desc.vres, 64, replace=False).astype(np.int32)
    wts = np.random.default_rng(9).choice([-1.0, 1.0], 64)
    _, _, _, gv = O.depth(osen, pos, R, res, org, val, scale=2.0, bias=0.5, pixels=pix,
                          grad_depth=wts)
    top = np.argsort(-np.abs(gv).reshape(-1))[:12]
    h = 1e-3
    for flat in top:
        li, l = divmod(int(flat), 512)
        v2 = val.copy()
        v2[li, l] += h
        Dp, _, _, _ = O.depth(osen, pos, R, res, org, v2, scale=2.0, bias=0.5, pixels=pix, want_grad=False)
        v2[li, l] -= 2 * h
        Dm, _, _, _ = O.depth(osen, pos, R, res, org, v2, scale=2.0, bias=0.5, pixels=pix, want_grad=False)
        fd = float(((Dp - Dm) / (2 * h) * wts).sum())
        # values are float32: the perturbation is what float32 can represent
        assert abs(fd - gv[li, l]) <= 2e-3 * abs(gv[li, l]) + 1e-7, (li, l, fd, gv[li, l])


def test_ending_walks_at_low_transmittance_changes_nothing_measurable():
    """What the GPU kernels' early end (each ray's walk stops once its transmittance is below
    1e-9) changes, measured on the FP64 definition: the depths by at most 1e-9 x the range
    (the bound the kernels rely on), the pose and log-odds gradients by far less than the
    GPU tests' tolerances (1e-5 / 1e-4 of the largest)."""
    spec, desc, frames, osen, res, org, val = _small_map()
    pos, R = _perturbed(frames)
    rng = np.random.default_rng(9)
    pix = rng.choice(desc.hres * desc.vres, 2000, replace=False).astype(np.int32)
    gd = rng.choice([-1.0, 1.0], len(pix))
    for scale, bias in ((4.0, 0.0), (12.0, 0.0), (1.0, -1.0)):
        full = O.depth(osen, pos, R, res, org, val, scale=scale, bias=bias, pixels=pix,
                       grad_depth=gd)
        cut = O.depth(osen, pos, R, res, org, val, scale=scale, bias=bias, pixels=pix,
                      grad_depth=gd, stop_transmittance=1e-9)
        assert np.abs(full[0] - cut[0]).max() <= 1e-9 * desc.max_range + 1e-15, scale
        g_full = (full[1] * gd[:, None]).sum(axis=0)
        g_cut = (cut[1] * gd[:, None]).sum(axis=0)
        for blk in (slice(0, 3), slice(3, 6)):
            assert np.abs(g_full[blk] - g_cut[blk]).max() <= 1e-7 * np.abs(g_full[blk]).max()
        assert np.abs(full[3] - cut[3]).max() <= 1e-7 * np.abs(full[3]).max()
