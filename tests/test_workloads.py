"""The seeded synthetic worlds: deterministic, world-seeded, in the stated ranges."""

import math

from exact_ballpark_b200.workloads import FOLLOW, ORBIT, WARP, flight_worlds


def test_worlds_are_deterministic_and_per_world_seeded():
    a, b = flight_worlds(3, 8, 4), flight_worlds(3, 8, 4)
    assert a.rows == b.rows and a.target == b.target
    c = flight_worlds(3, 16, 4)
    assert c.rows[:32] == a.rows                       # world w's draw depends on (seed, w) only


def test_ranges_and_targets():
    w = flight_worlds(11, 200, 4)
    for i, r in enumerate(w.rows):
        assert all(abs(c) <= 5e4 for c in r["pos"])
        assert 100.0 <= r["max_vel"] <= 3000.0 + 1e-9
        assert 1e6 <= r["mass"] <= 1e9 + 1e-3
        assert 0.1 <= r["agility"] <= 5.0 and 20.0 <= r["radius"] <= 500.0
        if w.follow_mask[i] or w.orbit_mask[i]:
            t = w.target[i]
            assert t // 4 == i // 4 and t != i and 500.0 <= w.range_[i] <= 30000.0
        else:
            assert w.warp_mask[i] and 3000 <= w.warp_factor[i] <= 10000
            d = math.dist(w.point[i], r["pos"])
            assert 1e8 * 0.99 <= d <= 1e11 * 1.01
    kinds = sum(w.follow_mask), sum(w.orbit_mask), sum(w.warp_mask)
    assert all(k > 150 for k in kinds)


def test_partition_workloads_carry_every_column_the_park_loads():
    """The partition workloads (the ragged headline's worlds and the reference's space benchmark shape) give every
    column VecModesPark.load_columns takes, each as the same worlds given as rows would load it."""
    import numpy as np

    from exact_ballpark_b200.modes import ROW_COLUMNS, rows_to_columns
    from exact_ballpark_b200.workloads import face_worlds, partition_worlds
    keys = [k for k, _, _ in ROW_COLUMNS] + ["pos", "vel"]
    for pw in (face_worlds(1, 16), partition_worlds(1, 16)):
        assert set(keys) <= set(pw.cols), sorted(set(keys) - set(pw.cols))
        rows = [{k: (pw.cols[k][i].tolist() if k in ("pos", "vel") else pw.cols[k][i].item()) for k in keys}
                for i in range(pw.n)]
        back = rows_to_columns(rows)
        for k in keys:
            assert np.array_equal(back[k], np.asarray(pw.cols[k]).astype(back[k].dtype)), k
