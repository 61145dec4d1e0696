"""The CPU oracle (oracle/flight.cpp's tick, oracle/park.py's commands) against the golden traces recorded on the
reference (tests/golden/trace.py): every tick's state digest of every scenario, bit for bit. Pins the oracle that
the GPU tests then use as their checker on inputs beyond the fixtures."""

import numpy as np
import pytest

import trace as tr
from golden_util import GOLDEN, available_traces
from oracle.park import OraclePark


def replay_oracle(t: dict):
    ctor = dict(t["ctor"])
    park = OraclePark(ctor.pop("n"), **ctor)
    bad = []

    def on_tick(k, p):
        mm = tr.first_mismatch(t, k, tr.field_digests(p))
        if mm and not bad:
            bad.append((k, mm))
    tr.replay(t, park, on_tick=on_tick)
    return park, bad


@pytest.mark.parametrize("name", available_traces())
def test_oracle_replays_the_golden_trace(name):
    groups = tr.load(GOLDEN / name)
    failures = []
    for gi, t in enumerate(groups):
        park, bad = replay_oracle(t)
        if bad:
            failures.append((gi, t["ctor"], bad[0]))
        else:
            for f, want in t["final"].items():
                got = tr.canonical(getattr(park, f))
                assert np.array_equal(got.view(np.uint64) if got.dtype == np.float64 else got,
                                      want.view(np.uint64) if want.dtype == np.float64 else want), (name, gi, f)
    assert not failures, f"{len(failures)} of {len(groups)} parks differ; first: {failures[:3]}"


def test_a_planted_fault_in_the_oracle_is_caught():
    """A perturbed state (one position one ulp off before the first tick) makes the digests differ: the replay check
    can fail."""
    t = tr.load(GOLDEN / "trace_w0_nodo_new")[0]
    ctor = dict(t["ctor"])
    park = OraclePark(ctor.pop("n"), **ctor)
    bad = []
    first = [True]

    def tick():
        if first[0]:
            park.pos[5, 0] = np.nextafter(park.pos[5, 0], np.inf)
            first[0] = False
        park.evolve()

    def on_tick(k, p):
        mm = tr.first_mismatch(t, k, tr.field_digests(p))
        if mm and not bad:
            bad.append((k, mm))
    tr.replay(t, park, tick=tick, on_tick=on_tick)
    assert bad and "pos" in bad[0][1]
