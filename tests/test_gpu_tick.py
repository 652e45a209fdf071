"""Batched ticks: every agent's labels and the shared map match solo runs bit for bit."""
import numpy as np
import pytest

from nanomap_b200 import _native as N
from nanomap_b200 import api as A
from nanomap_b200 import scenes as S
from oracle import oracle as O
from tests.workloads import compare_labels, compare_maps, oracle_frame

pytestmark = pytest.mark.gpu


def _agents(ctx, n_agents=6, seed=3):
    """Uneven sensors (three frustum shapes and a spinning range sensor) in the small world."""
    import torch
    spec = S.SCENES["plain_small"]
    scene = S.make_scene(spec, 1)
    sim = A.SimMap(ctx, 0.05, boxes=scene.boxes, cylinders=scene.cylinders, vox_min=(0, 0, 0),
                   vox_max=(400, 400, 100))
    shapes = [(320, 240, 5.0, 87, 58), (640, 480, 10.0, 87, 58), (1280, 720, 8.0, 87, 58)]
    sensors, agents = [], []
    for a in range(n_agents):
        if a == n_agents - 1:
            d = A.sensor_desc(type=N.NM_SENSOR_LASER, hres=1024, vres=64, hfov_deg=360.0, vfov_deg=30.0,
                              max_range=20.0, explicit_log_odds=1, log_odds_hit=0.85, log_odds_miss=-0.4,
                              frame_transform=S.OPTICAL_TO_BODY)
        else:
            w, h, r, hf, vf = shapes[a % 3]
            d = A.sensor_desc(type=0, hres=w, vres=h, hfov_deg=hf, vfov_deg=vf, max_range=r,
                              explicit_log_odds=1, log_odds_hit=0.85, log_odds_miss=-0.4,
                              frame_transform=S.OPTICAL_TO_BODY)
        s = A.Sensor(ctx, d)
        sensors.append(s)
        traj = S.trajectory(scene, 4, seed=seed + 17 * a)
        rng = [torch.zeros(d.vres, d.hres, device="cuda") for _ in traj]
        for (p, q), r in zip(traj, rng):
            sim.render(s, A.Pose(p, q), r)
        agents.append([(A.Pose(p, q), r) for (p, q), r in zip(traj, rng)])
    return sim, sensors, agents


def test_tick_labels_match_solo_runs(ctx):
    sim, sensors, agents = _agents(ctx)
    n = len(sensors)
    m = A.Map(ctx, A.map_desc(res=0.05, max_agents=n))
    frames = [(sensors[a], agents[a][0][0], agents[a][0][1], a) for a in range(n)]
    m.tick(frames, flags=N.NM_DEFER_INTEGRATE)
    for a in range(n):
        solo = A.Map(ctx, A.map_desc(res=0.05))
        solo.insert_ranges(sensors[a], agents[a][0][0], agents[a][0][1], flags=N.NM_DEFER_INTEGRATE)
        errs = compare_labels(m.export_labels(a), solo.export_labels(0))
        assert not errs, f"agent {a}: " + "; ".join(errs[:3])
        solo.close()
    m.integrate()


@pytest.mark.parametrize("variant", ["down_always", "nearest_crossing"])
def test_tick_map_equals_sequential_solo(ctx, variant):
    """The shared map after ticks equals inserting every agent's frame in agent order (both
    roundings; the clamp-on-crossing order with thresholds outside the clamp range)."""
    sim, sensors, agents = _agents(ctx)
    n = len(sensors)
    kw = dict(res=0.05)
    if variant == "nearest_crossing":
        kw.update(rounding=N.NM_ROUND_NEAREST, clamp_mode=N.NM_CLAMP_ON_CROSSING, clamp_min=-1.0,
                  clamp_max=1.5, thres_hit=1.6, thres_miss=-1.1)
    batched = A.Map(ctx, A.map_desc(max_agents=n, **kw))
    sequential = A.Map(ctx, A.map_desc(**kw))
    for t in range(3):
        batched.tick([(sensors[a], agents[a][t][0], agents[a][t][1], a) for a in range(n)])
        for a in range(n):
            sequential.insert_ranges(sensors[a], agents[a][t][0], agents[a][t][1])
    errs = compare_maps(batched.export(), sequential.export())
    assert not errs, "; ".join(errs[:5])
    sb, ss = batched.stats(), sequential.stats()
    assert sb["visits"] == ss["visits"] and sb["error_flags"] == 0


def test_tick_plan_graph_replay_matches_sequential(ctx, tmp_path):
    """Plans render from the sim map inside the graph; results equal the solo pipeline."""
    import torch
    sim, sensors, agents = _agents(ctx, n_agents=4)
    n = len(sensors)
    bufs = [torch.zeros(s.desc.vres, s.desc.hres, device="cuda") for s in sensors]
    planned = A.Map(ctx, A.map_desc(res=0.05, max_agents=n))
    plan = A.TickPlan(planned, [(sensors[a], bufs[a], a) for a in range(n)], sim=sim)
    best, us = plan.autotune(str(tmp_path / "tune.txt"))
    assert best[0] * best[1] in (64, 128) or (best[0] * best[1]) % 256 == 0
    assert (tmp_path / "tune.txt").read_text().strip()
    best2, _ = plan.autotune(str(tmp_path / "tune.txt"))  # served from the cache
    assert best2 == best
    sequential = A.Map(ctx, A.map_desc(res=0.05))
    scratch = torch.zeros(1280 * 720, device="cuda")
    for t in range(3):
        for a in range(n):
            plan.set_pose(a, agents[a][t][0])
        plan.run()
        for a in range(n):
            d = sensors[a].desc
            r = scratch[: d.vres * d.hres].view(d.vres, d.hres)
            sim.render(sensors[a], agents[a][t][0], r)
            sequential.insert_ranges(sensors[a], agents[a][t][0], r)
    torch.cuda.synchronize()
    errs = compare_maps(planned.export(), sequential.export())
    assert not errs, "; ".join(errs[:5])
    plan.close()


def test_tick_rejects_bad_slots(ctx):
    import torch
    desc = A.sensor_desc(hres=32, vres=32, max_range=5.0)
    s = A.Sensor(ctx, desc)
    m = A.Map(ctx, A.map_desc(res=0.1, max_agents=2))
    r = torch.zeros(32, 32, device="cuda")
    with pytest.raises(N.NanomapError):
        m.tick([(s, A.Pose((0, 0, 1), (1, 0, 0, 0)), r, 2)])
    with pytest.raises(N.NanomapError):
        m.tick([(s, A.Pose((0, 0, 1), (1, 0, 0, 0)), r, 0)] * 33)


def test_sixteen_agent_plan_ticks_match_solo_sequential_and_oracle(ctx):
    """The batched tick at its full size: 16 agents of uneven sensors (6 x 320x240 at 5 m,
    6 x 640x480 at 10 m, 3 x 1280x720 at 8 m, one spinning 64 x 1024 at 20 m) in the 20 x 20 x 5
    m world at 0.05 m, rendered with range noise and labelled by one graph-replayed tick plan per
    tick.  Every tick, every agent's label plane equals its solo insert of the same ranges bit
    for bit, and the spinning sensor's labels equal the oracle's; after the ticks the shared map
    equals the agents' frames inserted one by one in agent order."""
    import torch
    spec = S.SCENES["plain_small"]
    scene = S.make_scene(spec, 1)
    lo, hi = S.tick_sim_box(spec)
    sim = A.SimMap(ctx, S.TICK_RES, boxes=scene.boxes, cylinders=scene.cylinders, vox_min=lo,
                   vox_max=hi)
    sensors = [A.Sensor(ctx, A.sensor_desc(**S.tick_agent_desc_kwargs(a))) for a in S.TICK_AGENTS]
    n = len(sensors)
    assert n == 16
    ticks = 3
    trajs = [[A.Pose(p, q) for p, q in S.trajectory(scene, ticks, seed=101 + 37 * a)]
             for a in range(n)]
    bufs = [torch.zeros(s.desc.vres, s.desc.hres, device="cuda") for s in sensors]
    kw = dict(res=S.TICK_RES, initial_leaf_capacity=1 << 20)
    mb = A.Map(ctx, A.map_desc(max_agents=n, **kw))
    plan = A.TickPlan(mb, [(sensors[a], bufs[a], a) for a in range(n)], sim=sim)
    plan.set_noise(0.005, 0.02, 99)
    seq = A.Map(ctx, A.map_desc(**kw))
    solo = A.Map(ctx, A.map_desc(**kw))
    laser = n - 1
    assert sensors[laser].desc.type == N.NM_SENSOR_LASER
    osen = O.Sensor.from_desc(sensors[laser].desc)
    for t in range(ticks):
        for a in range(n):
            plan.set_pose(a, trajs[a][t])
        plan.run(flags=N.NM_DEFER_INTEGRATE)
        torch.cuda.synchronize()
        for a in range(n):
            solo.reset()
            solo.insert_ranges(sensors[a], trajs[a][t], bufs[a], flags=N.NM_DEFER_INTEGRATE)
            got = mb.export_labels(a)
            assert len(got[0]) > 0, f"tick {t} agent {a}: no labels"
            errs = compare_labels(got, solo.export_labels(0))
            assert not errs, f"tick {t} agent {a} vs solo: " + "; ".join(errs[:3])
            if a == laser:
                R, eye, mt = oracle_frame(sensors[a].desc, trajs[a][t], S.TICK_RES, N.NM_ROUND_DOWN)
                om = O.Map(S.TICK_RES, rounding=1)
                d = sensors[a].desc
                om.insert(R, eye, mt, d.log_odds_hit, d.log_odds_miss,
                          osen.points(bufs[a].cpu().numpy()), threads=8, keep_labels=True)
                errs = compare_labels(got, om.labels())
                assert not errs, f"tick {t} laser vs oracle: " + "; ".join(errs[:3])
        mb.integrate()
        for a in range(n):
            seq.insert_ranges(sensors[a], trajs[a][t], bufs[a])
    errs = compare_maps(mb.export(), seq.export())
    assert not errs, "; ".join(errs[:5])
    sb, ss = mb.stats(), seq.stats()
    assert sb["visits"] == ss["visits"] and sb["error_flags"] == 0 and ss["error_flags"] == 0
    plan.close()
