"""The composed park on the GPU, through the C ABI (ebb_composed_tick, ebb_composed_file) and the park's commands,
against the golden batches recorded on the reference's composed park (tests/golden/combat_trace.py with the
composed fields): the reference's composed scenarios with dynamical orientation (tests/park_cases.py; seed 1
development, seed 2 held out: ship clusters with fixed spheres meeting by the gradient method, FOLLOW and ORBIT at short
range, warps into the cluster dropping out among the others, the setters that re-file, cloaks, formations, missiles
launched at the ships): every field's digest after every step over the rows holding a ball (the collision
acceleration, the partition's filing and the collision list included), the DoCollision events and the
ReserveFormationSlot answers, bit for bit."""

import pytest
import torch

import combat_trace as ct

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")]


@pytest.mark.parametrize("seed", [1, 2], ids=["development", "held_out"])
def test_the_gpu_composed_park_replays_the_golden_batches(seed):
    from exact_ballpark_b200 import VecComposedPark
    formations, batches = ct.load(ct.GOLDEN / f"composed_{seed}")
    failures = []
    for bi, b in enumerate(batches):
        p, where = ct.make_park(VecComposedPark, b["cfg"], formations, "cuda")
        bad = ct.replay(p, b, where, fields=ct.COMPOSED_FIELDS)
        p.check()
        if bad:
            failures.append((bi, bad[:2]))
    assert not failures, f"{len(failures)} of {len(batches)} batches differ, first {failures[:2]}"
