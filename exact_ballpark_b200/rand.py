"""glibc's rand() on the device, one generator a world (include/ebb.h: ebb_glibc_srand, ebb_glibc_rand): destiny's
floatrand source for shuffled proximity sensors (the reference's exact_ballpark/glibc_rand.py GlibcRandom and
vec_space.py's glibc_srand). A world's state is an int32 row of RAND_WORDS (the table, then the two indices)."""

from __future__ import annotations

import torch

from . import _native

RAND_WORDS = 33
RAND_MAX = 2147483647.0


def srand(seeds: torch.Tensor) -> torch.Tensor:
    """srand(seed) for each world: the states [W, RAND_WORDS] int32 on the seeds' device."""
    seeds = seeds.to(torch.int64).contiguous()
    state = torch.empty(seeds.numel(), RAND_WORDS, dtype=torch.int32, device=seeds.device)
    with torch.cuda.device(seeds.device):
        rc = _native.lib().ebb_glibc_srand(seeds.data_ptr(), seeds.numel(), state.data_ptr(),
                                           torch.cuda.current_stream(seeds.device).cuda_stream)
    _native.check(rc, "ebb_glibc_srand")
    return state


def rand(state: torch.Tensor, draws: int) -> torch.Tensor:
    """`draws` values of rand() for each world [W, draws] int32, the states advanced in place."""
    out = torch.empty(state.shape[0], int(draws), dtype=torch.int32, device=state.device)
    with torch.cuda.device(state.device):
        rc = _native.lib().ebb_glibc_rand(state.data_ptr(), state.shape[0], int(draws), out.data_ptr(),
                                          torch.cuda.current_stream(state.device).cuda_stream)
    _native.check(rc, "ebb_glibc_rand")
    return out


def floatrand(state: torch.Tensor, draws: int = 1) -> torch.Tensor:
    """destiny's floatrand (Ball.cpp:19): rand() / RAND_MAX as a double, [W, draws] (a tensor divisor: torch on CUDA
    divides by a Python number through its reciprocal, which is not the IEEE quotient)."""
    r = rand(state, draws).to(torch.float64)
    return r / torch.tensor(RAND_MAX, dtype=torch.float64, device=r.device)
