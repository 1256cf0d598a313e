"""hp_Deposit_noalloc against hp_Deposit, through the C ABI.

hp_Deposit_noalloc serves callers that cannot let the library allocate GPU
memory (hosts that pool or budget every device byte themselves, or loops that
must not pay cudaMalloc's device synchronisation): it keeps its per-cell
scratch in one fixed array inside the library and writes into the caller's
buffer.  Its densities must equal hp_Deposit's (both use the same lane sums,
warp trees and node gather, so the tolerance here is zero) on consecutive
calls, with the shared scratch reused between them.  The file name sorts
last so that a stop-at-first-failure run has run every other test first.
"""
import ctypes as C

import numpy as np
import pytest

import hpic
from hpic.decks import ccp_deck

pytestmark = pytest.mark.gpu


def noalloc_density(case):
    import torch
    out = torch.full((case.info.nsp * case.info.Gsize,), float("nan"), dtype=torch.float64, device="cuda")
    hpic._check(hpic.lib().hp_Deposit_noalloc(case.h, C.c_void_p(out.data_ptr()), None))
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_noalloc_deposit_matches_deposit_twice():
    deck = ccp_deck(65, 33, 0.02, 0.01, ppc=24, voltage=150.0)
    case = hpic.Case(deck, seed=31)
    for round_ in range(2):
        case.step(3)
        case.Deposit()
        ref = case.grid("DEN")
        got = noalloc_density(case)
        assert got.shape == ref.shape
        assert np.array_equal(got.view(np.uint64), ref.view(np.uint64)), f"call {round_ + 1} differs"
    # a second, smaller case reuses the same scratch right after
    small = hpic.Case(ccp_deck(17, 9, 0.005, 0.0025, ppc=10), seed=5)
    small.Deposit()
    assert np.array_equal(noalloc_density(small).view(np.uint64), small.grid("DEN").view(np.uint64))


def test_noalloc_rejects_batched_cases_and_keeps_the_current_device():
    import torch
    cases = [hpic.Case(ccp_deck(17, 9, 0.005, 0.0025, ppc=8), seed=s) for s in (3, 4)]
    batch = hpic.Batch(cases)
    with pytest.raises(hpic.HpicError) as e:
        hpic._check(hpic.lib().hp_Deposit_noalloc(cases[0].h, C.c_void_p(1), None))
    assert e.value.status == hpic.HP_ERR_ARG
    batch.close()
    dev = torch.cuda.current_device()
    alone = hpic.Case(ccp_deck(17, 9, 0.005, 0.0025, ppc=8), seed=6)
    alone.Deposit()
    noalloc_density(alone)
    assert torch.cuda.current_device() == dev


def test_noalloc_rejects_cases_beyond_the_scratch():
    # 1027 x 257 nodes: 2 x 1026 x 256 = 525312 (species x cells) > 2^19; the
    # check runs before any device work, so a light load is enough
    big = hpic.Case(ccp_deck(1027, 257, 0.32, 0.08, ppc=1), seed=2)
    with pytest.raises(hpic.HpicError) as e:
        hpic._check(hpic.lib().hp_Deposit_noalloc(big.h, C.c_void_p(1), None))
    assert e.value.status == hpic.HP_ERR_CAPACITY
