"""hp_profile_step: per-kernel device times of op-by-op steps.  The steps it
runs are the case's real steps (the state equals that of hp_step), every
kernel of the step appears with its launches, and bad arguments are
refused."""
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(REPO, "hybrid-final_b200"))

import hpic  # noqa: E402
from hpic.decks import ccp_deck  # noqa: E402


def test_arguments_are_checked_without_a_gpu():
    L = hpic.lib()
    n = hpic.C.c_int(0)
    assert L.hp_profile_step(None, 1, None, None, 0, hpic.C.byref(n)) == hpic.HP_ERR_ARG


@pytest.mark.gpu
@pytest.mark.parametrize("field_mode", [1, 2])
def test_profile_steps_are_real_steps(field_mode):
    deck = ccp_deck(65, 33, 0.02, 0.01, ppc=12, voltage=150.0, max_np_factor=8)
    a = hpic.Case(deck=deck, seed=9, field_mode=field_mode)
    b = hpic.Case(deck=deck, seed=9, field_mode=field_mode)
    stats = a.profile(3)
    b.step(3)
    names = {n: (l, ms) for n, l, ms in stats}
    for k in ("k_advance", "k_move", "k_sort_push", "k_sort_count", "k_mcc_ar", "k_deposit_cells",
              "k_deposit_nodes", "k_potential", "k_efield", "k_accumulate"):
        assert names[k][0] == 3 and names[k][1] > 0, k
    assert ("k_pcg" in names) == (field_mode == 1)
    assert ("k_gemm" in names) == (field_mode == 2)
    assert a.tstep() == b.tstep() == 3
    for s in range(a.info.nsp):
        ga, xa = a.particles(s)
        gb, xb = b.particles(s)
        assert np.array_equal(ga, gb)
        for u, v in zip(xa, xb):
            assert np.array_equal(u.view(np.uint32), v.view(np.uint32))
    assert np.array_equal(a.grid("PHI").view(np.uint32), b.grid("PHI").view(np.uint32))
    # after a profile the graph path continues from the same state
    a.step(2)
    b.step(2)
    assert np.array_equal(a.grid("AVE_PHI").view(np.uint64), b.grid("AVE_PHI").view(np.uint64))
