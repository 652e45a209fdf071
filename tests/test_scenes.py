"""Seeded synthetic scenes are deterministic and trajectories stay in free space."""
import numpy as np

from nanomap_b200 import scenes as S


def test_splitmix_reference_values():
    # splitmix64 with seed 0: the first outputs of the published generator
    z = S.splitmix64(0, 3)
    assert [int(v) for v in z] == [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F]


def test_scene_is_deterministic():
    a = S.make_scene("sim_headline", 3)
    b = S.make_scene("sim_headline", 3)
    c = S.make_scene("sim_headline", 4)
    assert np.array_equal(a.boxes, b.boxes) and np.array_equal(a.cylinders, b.cylinders)
    assert not np.array_equal(a.boxes, c.boxes)
    assert a.boxes.shape == (2000, 6) and a.cylinders.shape == (300, 5)
    e = a.boxes[:, 3:] - a.boxes[:, :3]
    assert e.min() >= 0.1 and e.max() <= 3.0
    assert a.cylinders[:, 2].min() >= 0.05 and a.cylinders[:, 2].max() <= 0.5
    assert a.vox_max == (800, 800, 200)


def test_trajectory_in_free_space():
    sc = S.make_scene("plain_small", 1)
    tr = S.trajectory(sc, 10, seed=7)
    assert len(tr) == 10
    for pos, q in tr:
        assert not S.occupied(sc, pos, 0.0)
        assert abs(sum(v * v for v in q) - 1.0) < 1e-12
    steps = [np.linalg.norm(np.subtract(tr[i + 1][0], tr[i][0])) for i in range(9)]
    assert all(abs(s - 0.2) < 1e-9 or s < 1e-12 for s in steps)


def test_analytic_box_ranges_equal_the_oracle():
    """The bench's exact ray-box ranges (numpy, FP64) equal the oracle's renderer bit for bit."""
    from nanomap_b200 import api as A
    from oracle import oracle as O
    spec = S.SCENES["plain_small"]
    scene = S.make_scene(spec, 1)
    desc = A.sensor_desc(**S.sensor_desc_kwargs(spec))
    for pos, q in S.trajectory(scene, 9, seed=7)[::4]:
        _, _, _, pm = A.frame_params(desc, A.Pose(pos, q), spec.map_res, 1)
        got = S.analytic_box_ranges(scene, pm, spec.width, spec.height, spec.max_range, pos, q)
        ref = O.render_boxes(O.Sensor.from_desc(desc), pos, S.rotation_matrix(q), scene.boxes)
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_tick_agents_are_the_sixteen_uneven_sensors():
    kinds = [(a[0], a[1], a[2], a[5]) for a in S.TICK_AGENTS]
    assert len(kinds) == 16
    assert kinds.count((0, 320, 240, 5.0)) == 6 and kinds.count((0, 640, 480, 10.0)) == 6
    assert kinds.count((0, 1280, 720, 8.0)) == 3 and kinds.count((1, 1024, 64, 20.0)) == 1


def test_bench_map_and_label_comparisons():
    import bench
    o = np.array([[0, 0, 0], [8, 0, 0]], np.int32)
    v = np.zeros((2, 512), np.float32)
    v[1, 3] = 0.85
    a = np.zeros((2, 16), np.uint32)
    a[1, 0] = 8
    assert bench.maps_equal((o, v, a), (o[::-1], v[::-1], a[::-1]))
    assert bench.maps_equal((o, v, a), (o[1:], v[1:], a[1:]))  # an all-zero leaf may be absent
    v2 = v.copy()
    v2[1, 3] = np.float32(0.85) + np.float32(1e-7)
    assert not bench.maps_equal((o, v, a), (o, v2, a))
    w = np.zeros((2, 32), np.uint32)
    w[0, 17] = 1
    assert bench.labels_equal((o, w), (o[::-1], w[::-1]))
    assert not bench.labels_equal((o, w), (o[1:], w[1:]))
