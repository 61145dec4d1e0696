"""The server layer's torch path (exact_ballpark_b200.server) on the CPU over the CPU oracle's flight park
(oracle/server_view.py), against the golden ticks recorded on the reference's own server layer: the reference's server
scenarios without and with dynamical orientation, its pending-query scenarios and its OnTick scenarios, every park
field, the update batch, the answers and what every client is sent, after every tick. The layer's logic is held to the
reference without a GPU; the GPU tests hold both of its paths over the GPU park to the same goldens."""

import pytest

import server_trace as st


def _oracle_park(n, friction=1.0e6, tick_interval_ms=1000, device="cpu", dynamical_orientation=False):
    from oracle.park import OraclePark
    from oracle.server_view import OracleParkView
    return OracleParkView(OraclePark(n, friction=friction, tick_interval_ms=tick_interval_ms,
                                     dynamical_orientation=dynamical_orientation))


@pytest.mark.parametrize("name,run", [("server_modes", 0), ("server_modes", 1), ("server_modes_do", 0),
                                      ("server_modes_do", 1), ("server_pending", 0), ("server_pending", 1),
                                      ("server_ontick", 0), ("server_ontick", 1), ("server_ontick", 2),
                                      ("server_ontick", 3)])
def test_the_torch_path_over_the_oracle_park_replays_the_golden_ticks(name, run):
    from exact_ballpark_b200 import server
    r = st.load(st.GOLDEN / name)[run]
    bad = st.replay(server, _oracle_park, r, "cpu", kernel="torch")
    assert not bad, f"{len(bad)} differences, first {bad[:3]}"


def _oracle_collide_park(worlds, slots, friction=1.0e6, tick_interval_ms=1000, device="cpu"):
    from oracle.collide_park import OracleCollidePark
    from oracle.server_view import OracleParkView
    return OracleParkView(OracleCollidePark(worlds, slots, friction=friction, tick_interval_ms=tick_interval_ms))


@pytest.mark.parametrize("name,run", [("server_collide", 0), ("server_collide", 1), ("server_collide_ontick", 0)])
def test_the_collision_parks_layer_over_the_oracle_replays_the_golden_ticks(name, run):
    from exact_ballpark_b200 import server
    r = st.load(st.GOLDEN / name)[run]
    bad = st.replay(server, _oracle_collide_park, r, "cpu")
    assert not bad, f"{len(bad)} differences, first {bad[:3]}"
