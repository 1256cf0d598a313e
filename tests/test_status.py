"""Every bit of the device status word, forced from the host.

The reference has no error reporting: a CUDA error calls exit()
(src/cuda_main.cu:2-9) and an overfull cell is halved in place by ReArgPtcls
(src/cuda_Sortboundary.cu:23-40).  Here the kernels set a bit of the case's
status word and carry on with defined results; each test drives one
condition with ordinary inputs and checks the bit.  HP_STATUS_WAIT_TIMEOUT is
never raised: no kernel of this library spins on a flag (the cluster
barriers are cluster.sync())."""
import numpy as np
import pytest

import hpic
from hpic.decks import ccp_deck, dielectric_deck

pytestmark = pytest.mark.gpu


def stepped_status(case, n=1):
    case.step(n)
    return case.status()


def test_cell_overflow():
    # 31 particles per cell in 64 slots load (a load past half the slots is
    # refused at creation); the first step's sort gathers up to 40 in a cell,
    # past the reference's ReArg condition (2 x count > slots), which the
    # next Move checks (src/cuda_Sortboundary.cu:63-65 checks it on entry)
    c = hpic.Case(ccp_deck(17, 9, 0.005, 0.0025, ppc=31), seed=1, cap_per_cell=64, move_mode=1)
    assert c.status() == 0
    assert stepped_status(c, 2) & hpic.STATUS_CELL_OVERFLOW
    # the same case with room runs clean
    ok = hpic.Case(ccp_deck(17, 9, 0.005, 0.0025, ppc=31), seed=1, cap_per_cell=128, move_mode=1)
    assert stepped_status(ok, 3) == 0
    with pytest.raises(hpic.HpicError) as e:
        hpic.Case(ccp_deck(17, 9, 0.005, 0.0025, ppc=40), seed=1, cap_per_cell=64)
    assert e.value.status == hpic.HP_ERR_CAPACITY


@pytest.mark.parametrize("field_mode,kw", [(0, dict(pcg_max_iter=1)), (1, dict(pcg_max_iter=1)),
                                           (2, dict(fs_passes=1, pcg_rtol=1e-14))])
def test_field_no_convergence(field_mode, kw):
    c = hpic.Case(ccp_deck(33, 17, 0.01, 0.005, ppc=10), seed=2, field_mode=field_mode, **kw)
    assert stepped_status(c) & hpic.STATUS_PCG_NOCONV


@pytest.mark.parametrize("field_mode", [0, 1, 2])
def test_nonfinite_field(field_mode):
    c = hpic.Case(ccp_deck(33, 17, 0.01, 0.005, ppc=10), seed=3, field_mode=field_mode)
    c.step(1)
    assert c.status() == 0
    b = c.grid("PCG_B")
    b[b.size // 2] = np.nan
    c.set_grid("PCG_B", b)
    assert stepped_status(c) & hpic.STATUS_NONFINITE


def test_walk_bound():
    # one electron at 1e15 m/s: its walk would cross ~1e9 cells in a step
    c = hpic.Case(ccp_deck(33, 17, 0.01, 0.005, ppc=10), seed=4, move_mode=1)
    counts, a = c.particles(0)
    a[2][a[0].size // 2] = 1e15
    c.set_particles(0, counts, *a)
    assert stepped_status(c) & hpic.STATUS_WALK_BOUND
    _, a1 = c.particles(0)
    assert np.abs(a1[2]).max() < 1e10, "the runaway electron was absorbed"


def test_surface_queue_overflow():
    # every electron sent down into the dielectric slab at 3e7 m/s (up to ~18
    # cells a step): more crossings than the case's queue holds
    c = hpic.Case(dielectric_deck(ppc=24), seed=5, cap_per_cell=64, move_mode=1)
    counts, a = c.particles(0)
    a[3][:] = -3e7
    c.set_particles(0, counts, *a)
    assert stepped_status(c) & hpic.STATUS_SURFACE_OVERFLOW


def test_served_request_retires_with_its_status_and_the_others_are_unchanged():
    """One request overflows its cells (62 particles per cell in 128 slots
    load; its first push gathers up to 80 in a cell); it retires with
    HP_STATUS_CELL_OVERFLOW and the requests it shared the device with return
    what they return alone, bit for bit."""
    from test_serve import OPTS, REQS, alone
    srv = hpic.Server(max_slots=3, steps_per_launch=7, **OPTS)
    good = [srv.submit(d, n, seed) for d, n, seed in REQS[:3]]
    bad = srv.submit(ccp_deck(17, 9, 0.005, 0.0025, ppc=62), 20, 99)
    res = {r.request_id: (r, den, phi) for r, den, phi in srv.run()}
    srv.close()
    assert res[bad][0].error == 0 and res[bad][0].status & hpic.STATUS_CELL_OVERFLOW
    for rid, (deck, nsteps, seed) in zip(good, REQS[:3]):
        r, den, phi = res[rid]
        assert r.error == 0 and r.status == 0
        d0, p0, _ = alone(deck, nsteps, seed)
        assert np.array_equal(den.view(np.uint64), d0.view(np.uint64))
        assert np.array_equal(phi.view(np.uint64), p0.view(np.uint64))
