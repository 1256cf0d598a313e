"""The served form (hp_server_*): continuous batching over resident cases.

Requests are admitted in arrival order as slots and device memory free up,
advanced together in batched rounds, and retired with their time-averaged
densities and potential.  A case's steps depend only on its own state, so
each result must equal, bit for bit, the same request run alone through
hp_case_create + hp_step, whatever it shared the device with and however
its steps were split into rounds."""
import numpy as np
import pytest

import hpic
from hpic.decks import ccp_deck

pytestmark = pytest.mark.gpu

REQS = [
    (ccp_deck(33, 17, 0.01, 0.005, ppc=12, voltage=150.0), 37, 11),
    (ccp_deck(17, 9, 0.005, 0.0025, ppc=10), 23, 12),
    (ccp_deck(65, 33, 0.02, 0.01, ppc=8, pressure_torr=0.1), 50, 13),
    (ccp_deck(33, 17, 0.01, 0.005, ppc=6, voltage=80.0), 9, 14),
    (ccp_deck(17, 9, 0.005, 0.0025, ppc=16, voltage=250.0), 61, 15),
]
OPTS = dict(field_mode=2, move_mode=1, gas_temp_mode=1, cap_per_cell=128)


def alone(deck, nsteps, seed):
    c = hpic.Case(deck, seed=seed, **OPTS)
    c.step(nsteps)
    n = c.average_count()
    den = c.grid("AVE_DEN").reshape(c.info.nsp, -1) / n
    phi = c.grid("AVE_PHI") / n
    pushes = c.pushes()
    c.close()
    return den, phi, pushes


def test_results_equal_alone_runs_in_any_mix():
    srv = hpic.Server(max_slots=3, steps_per_launch=7, **OPTS)
    ids = [srv.submit(d, n, seed) for d, n, seed in REQS]
    res = {r.request_id: (r, den, phi) for r, den, phi in srv.run()}
    srv.close()
    assert sorted(res) == sorted(ids)
    for rid, (deck, nsteps, seed) in zip(ids, REQS):
        r, den, phi = res[rid]
        assert r.error == 0 and r.status == 0 and r.steps == nsteps
        assert r.t_submit <= r.t_admit <= r.t_done
        d0, p0, pushes = alone(deck, nsteps, seed)
        assert r.particle_pushes == pushes
        assert np.array_equal(den.view(np.uint64), d0.view(np.uint64)), f"request {rid}: densities differ"
        assert np.array_equal(phi.view(np.uint64), p0.view(np.uint64)), f"request {rid}: potential differs"


def test_admission_respects_slots_and_budget():
    """With one slot the requests run one after another; a request larger than
    the whole budget is refused with HP_ERR_CAPACITY; a bad deck is reported,
    and neither stops the others."""
    srv = hpic.Server(max_slots=1, steps_per_launch=5, mem_budget_bytes=128 << 20, **OPTS)
    small = srv.submit(*REQS[1][:2], seed=3)
    bad = dict(REQS[1][0])
    bad["Geometry"] = dict(bad["Geometry"], SystemSpec=dict(bad["Geometry"]["SystemSpec"], NumGridx=1))
    nbad = srv.submit(bad, 5, seed=4)
    big = srv.submit(ccp_deck(257, 129, 0.08, 0.04, ppc=50), 5, seed=5)
    small2 = srv.submit(*REQS[3][:2], seed=6)
    res = {r.request_id: r for r, _, _ in srv.run()}
    srv.close()
    assert res[small].error == 0 and res[small2].error == 0
    assert res[nbad].error == hpic.HP_ERR_DECK
    assert res[big].error == hpic.HP_ERR_CAPACITY
    # one slot: the second small request was admitted after the first was done
    assert res[small2].t_admit >= res[small].t_done
