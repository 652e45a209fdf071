"""Optional torch binding of the expected-depth renderer: the test harness of its adjoint.

`ExpectedDepth.apply(values, xi, map, sensor, position, rotation, scale, bias)` renders the
expected depth (metres) of every pixel at the pose (position + rho, exp([phi]x) rotation),
xi = (rho, phi); its backward calls the library's adjoint for the gradients with respect to
the per-voxel log-odds (`values`, slot layout as `Map.values_copy`) and to xi.  The library's
native scan-to-map refinement (`Map.pose_refine`) needs none of this module.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from .api import Map, Sensor


def hat(v) -> np.ndarray:
    return np.array([[0.0, -v[2], v[1]], [v[2], 0.0, -v[0]], [-v[1], v[0], 0.0]])


def so3_exp(phi) -> np.ndarray:
    """Rodrigues' formula."""
    phi = np.asarray(phi, np.float64)
    th = float(np.linalg.norm(phi))
    K = hat(phi)
    if th < 1e-12:
        return np.eye(3) + K + 0.5 * K @ K
    return np.eye(3) + math.sin(th) / th * K + (1.0 - math.cos(th)) / th ** 2 * K @ K


def so3_left_jacobian(phi) -> np.ndarray:
    """J_l(phi): exp(phi + d) = exp(J_l(phi) d) exp(phi) to first order in d."""
    phi = np.asarray(phi, np.float64)
    th = float(np.linalg.norm(phi))
    K = hat(phi)
    if th < 1e-8:
        return np.eye(3) + 0.5 * K + K @ K / 6.0
    return (np.eye(3) + (1.0 - math.cos(th)) / th ** 2 * K
            + (th - math.sin(th)) / th ** 3 * K @ K)


class ExpectedDepth(torch.autograd.Function):
    @staticmethod
    def forward(ctx, values, xi, m: Map, sensor: Sensor, position, rotation, scale=1.0,
                bias=0.0):
        x = xi.detach().cpu().double().numpy()
        pos = np.asarray(position, np.float64) + x[:3]
        R = so3_exp(x[3:]) @ np.asarray(rotation, np.float64)
        vals = values.detach().contiguous()
        depth = m.depth_render(sensor, pos, R, values=vals, scale=scale, bias=bias)
        ctx.save_for_backward(vals, depth)
        ctx.args = (m, sensor, pos, R, x, scale, bias)
        return depth

    @staticmethod
    def backward(ctx, grad_depth):
        vals, depth = ctx.saved_tensors
        m, sensor, pos, R, x, scale, bias = ctx.args
        gv = torch.zeros_like(vals) if ctx.needs_input_grad[0] else None
        g = m.depth_backward(sensor, pos, R, grad_depth.contiguous(), values=vals,
                             grad_values=gv, scale=scale, bias=bias, depth=depth)
        # the adjoint differentiates with respect to a left increment at the evaluated pose;
        # chain through the exponential map to the coordinates of xi
        gx = np.concatenate([g[:3], so3_left_jacobian(x[3:]).T @ g[3:]])
        return gv, torch.from_numpy(gx), None, None, None, None, None, None


def expected_depth(values, xi, m: Map, sensor: Sensor, position, rotation, scale=1.0,
                   bias=0.0):
    return ExpectedDepth.apply(values, xi, m, sensor, position, rotation, scale, bias)
