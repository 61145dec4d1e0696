"""The server layer (exact_ballpark_b200.server) over the GPU flight park against the golden traces recorded on the
reference's own server layer (tests/golden/server_trace.py): the reference's server scenarios over the flight-mode
park, without and with dynamical orientation (seed 1 development, seed 2 held out; 40 worlds of one bubble each, 14
ticks of Actions calls: conflicting commands, duplicates dropped and kept, cloaks and uncloaks in both orders, local and
non-local SetBallPosition, follows and orbits of a cloaking ship, warps and warp-ins, every setter, refused values).
After every tick: every park field's digest and the update batch's digest (stamps, queued flags and rows, routes, the
uncloaks' recipients and the park's fields there, the bubble's additions, the narrowcast and character flags), bit for
bit. The CPU tests hold the queue's duplicate rule and the world lookup on a stand-in park."""

from types import SimpleNamespace

import pytest
import torch

import server_trace as st


def _golden(name):
    return st.load(st.GOLDEN / name)


@pytest.mark.gpu
@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")
@pytest.mark.parametrize("name", ["server_modes", "server_modes_do"], ids=["euler", "dynamical"])
@pytest.mark.parametrize("run", [0, 1], ids=["development", "held_out"])
def test_the_server_layer_replays_the_golden_ticks(name, run):
    from exact_ballpark_b200 import VecModesPark, server
    r = _golden(name)[run]
    bad = st.replay(server, VecModesPark, r, "cuda")
    assert not bad, f"{len(bad)} differences, first {bad[:3]}"


def test_the_server_goldens_hold_every_action_kind():
    from exact_ballpark_b200 import server
    for name in ("server_modes", "server_modes_do"):
        runs = _golden(name)
        assert len(runs) == 2
        kinds = {c[0] for r in runs for w in r["cases"] for t in w["ticks"] for c in t}
        assert {st.ACTION_KINDS[k] for k in kinds} <= set(server.CODE)
        assert len(kinds) >= 18
        for r in runs:
            T = len(r["cases"][0]["ticks"])
            assert r["park"].shape[0] == T and len(r["batch"]) == T


class _StandIn:
    """A park the server layer reads on the CPU: two worlds of three balls (ids 10, 11, 12 and 20, 21, 22)."""

    def __init__(self):
        from exact_ballpark_b200 import server
        self.dev = torch.device("cpu")
        self.R, self.W = 6, 2
        self.world = torch.tensor([0, 0, 0, 1, 1, 1])
        self.rows_of_world = torch.tensor([[0, 1, 2], [3, 4, 5]])
        self.ids_of_world = torch.tensor([[10, 11, 12], [20, 21, 22]])
        self.arange = torch.arange(6)
        self.kinds = frozenset(k for k in range(1, len(server.KINDS)) if k not in server.NOT_APPLIED)
        self.lookup = server.ModesAdapter.lookup.__get__(self)
        self.any_in_world = server.ModesAdapter.any_in_world.__get__(self)

    def clock(self):
        return torch.tensor([5, 5])


def test_push_drops_a_call_equal_to_the_worlds_last_and_keeps_the_rest():
    from exact_ballpark_b200 import server
    A = _StandIn()
    s = server.VecServer.__new__(server.VecServer)
    s.a, s.W, s.R, s.dev = A, A.W, A.R, A.dev
    s.settled = torch.tensor([True, False, False, True, True, True])
    s.slots = []
    s._reset_last()
    both = torch.tensor([True, True])
    a = s.push("SetMaxSpeed", both, torch.tensor([11, 22]), f=torch.tensor([[3.0], [float("nan")]]))
    assert a.ok.tolist() == [True, True] and a.row.tolist() == [1, 5]
    b = s.push("SetMaxSpeed", both, torch.tensor([11, 22]), f=torch.tensor([[3.0], [float("nan")]]))
    assert b.ok.tolist() == [False, True]          # the same call dropped; a NaN equals nothing
    c = s.push("SetMaxSpeed", both, torch.tensor([11, 23]), f=torch.tensor([[3.5], [1.0]]))
    assert c.ok.tolist() == [True, True] and c.row.tolist() == [1, -1]
    d = s.push("SetMaxSpeed", torch.tensor([True, False]), torch.tensor([11, 23]), f=torch.tensor([[3.0], [1.0]]))
    assert d.ok.tolist() == [True, False]          # not the last call any more: queued again
    e = s.push("CloakBall", both, torch.tensor([10, 24]), n=torch.tensor([1, 1]), f=torch.tensor([[9.0], [9.0]]))
    assert e.ok.tolist() == [True, False]          # not queued for a ball not in the park
    assert e.loc.tolist()[0] == 0                  # the bubble it was queued in
    f = s.push("CloakBall", both, torch.tensor([12, 21]), n=torch.tensor([1, 1]), f=torch.tensor([[9.0], [9.0]]))
    assert f.ok.tolist() == [True, True] and f.loc.tolist() == [-1, 0]
    g = s.push("FollowBall", both, torch.tensor([10, 20]), target=torch.tensor([12, 29]), f=torch.tensor([[5.0], [5.0]]))
    assert g.trow.tolist() == [2, -1]
    with pytest.raises(ValueError):
        s.push("LaunchMissile", both, torch.tensor([10, 20]))
    assert len(s.slots) == 7
    assert SimpleNamespace(**s.last).kind.tolist() == [server.CODE["FollowBall"]] * 2
