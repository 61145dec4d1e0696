"""The world-to-tile packing of the tiled schedule (host logic)."""

import torch

from exact_ballpark_b200.tiles import pack, plan_tiles, world_runs


def test_world_runs():
    assert world_runs(torch.tensor([0, 0, 1, 1, 1, 2])) == [0, 2, 5, 6]
    assert world_runs(torch.tensor([0, 1, 0])) is None                 # a world in two runs
    assert world_runs(torch.tensor([5, 5, 3, 3])) == [0, 2, 4]


def test_pack_keeps_worlds_whole_and_tiles_within_cap():
    runs = [0, 3, 10, 12, 20, 21, 40]
    for cap in (19, 20, 25, 40):
        rows = pack(runs, cap)
        assert rows[0] == 0 and rows[-1] == 40
        assert all(b - a <= cap for a, b in zip(rows[:-1], rows[1:]))
        assert set(rows) <= set(runs)


def test_plan_grows_the_cap_to_the_largest_world():
    w = torch.repeat_interleave(torch.arange(4), torch.tensor([3, 200, 5, 7]))
    p = plan_tiles(w, cap=128)
    assert p.cap >= 200 and p.block % 32 == 0 and p.block <= 256
    assert p.tile_rows[-1] == 215
    assert plan_tiles(torch.tensor([0, 1, 0])) is None
