"""The combat park on the GPU, through the C ABI (ebb_combat_tick) and the park's commands, against the golden
traces recorded on the reference's combat park (tests/golden/combat_trace.py): the reference's combat scenarios with
dynamical orientation (seed 1 development, seed 2 held out; missiles launched aimed and unaimed, at cloaked, removed
and warping targets, MissileFollow's refusals, formations reserved, followed, resized, left and freed, cloaks and
uncloaks, removals, velocity and massive setters, master and client, the missile exclusion of dynamical orientation
on and off): every field's digest after every step over the rows holding a ball, the DoCollision events and the
ReserveFormationSlot answers, bit for bit."""

import pytest
import torch

import combat_trace as ct

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")]


@pytest.mark.parametrize("seed", [1, 2], ids=["development", "held_out"])
def test_the_gpu_combat_park_replays_the_golden_batches(seed):
    from exact_ballpark_b200 import VecCombatPark
    formations, batches = ct.load(ct.GOLDEN / f"combat_{seed}")
    failures = []
    for bi, b in enumerate(batches):
        p, where = ct.make_park(VecCombatPark, b["cfg"], formations, "cuda")
        bad = ct.replay(p, b, where)
        p.check()
        if bad:
            failures.append((bi, bad[:2]))
    assert not failures, f"{len(failures)} of {len(batches)} batches differ, first {failures[:2]}"
