"""glibc's rand() after srand(seed): the CPU oracle (oracle/grand.py) and the device generator
(exact_ballpark_b200.rand, include/ebb.h: ebb_glibc_srand, ebb_glibc_rand) against the reference's own generator's
output (tests/golden/rand.npz: 40 seeds, edge seeds included, 2000 draws each, and the state after srand)."""

import numpy as np
import pytest
import torch

from golden_util import GOLDEN


def _golden():
    z = np.load(GOLDEN / "rand.npz")
    return z["seeds"], z["draws"], z["states"]


def test_the_oracle_draws_the_references_sequence():
    from oracle.grand import Rand
    seeds, draws, states = _golden()
    for i, sd in enumerate(seeds):
        g = Rand(int(sd))
        assert g.state() == states[i].tolist()
        assert [g.next() for _ in range(draws.shape[1])] == draws[i].tolist()


@pytest.mark.gpu
@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")
def test_the_device_generator_draws_the_references_sequence():
    from exact_ballpark_b200 import rand
    seeds, draws, states = _golden()
    st = rand.srand(torch.tensor(seeds, device="cuda"))
    assert (st.cpu().numpy().astype(np.int64) == states).all()
    got = torch.cat([rand.rand(st, 700), rand.rand(st, 1300)], dim=1)          # two calls: the state carries on
    assert (got.cpu().numpy().astype(np.int64) == draws).all()
    st2 = rand.srand(torch.tensor(seeds, device="cuda"))
    f = rand.floatrand(st2, 3).cpu().numpy()
    assert (f == draws[:, :3] / 2147483647.0).all()
