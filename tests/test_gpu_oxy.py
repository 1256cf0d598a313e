"""Ar/O2 and O2 reaction sets on the GPU vs. the CPU oracle, bit for bit.

Five species (e, Ar+, O2+, O+, O-), collision probabilities from the local
background, metastable and charged densities, attachment, detachment,
recombination, charge transfer between ion species and ionisation into
several species: the order of births, removals and hole filling is defined by
the library (mcc_oxy.cu) and restated by the oracle, so positions,
velocities, counts and per-channel tallies must agree exactly."""
import numpy as np
import pytest

import hpic
import oracle
from hpic.decks import ccp_deck

pytestmark = pytest.mark.gpu

OPTS = dict(field_mode=2, move_mode=1, gas_temp_mode=1)


def aro2_deck(ngx, ngy, xlen, ppc, volts=200.0):
    return ccp_deck(ngx, ngy, xlen, xlen / 2, gas="ArO2", ppc=ppc, pressure_torr=0.1, voltage=volts, te_ev=3.0,
                    ion_density={"Ar+": 1e15, "O2+": 2e14, "O+": 5e13, "O-": 2e14}, max_np_factor=8)


def o2_deck(ngx, ngy, xlen, ppc, volts=200.0):
    return ccp_deck(ngx, ngy, xlen, xlen / 2, gas="O2", ppc=ppc, pressure_torr=0.1, voltage=volts, te_ev=3.0,
                    ion_density={"O2+": 1e15, "O+": 1e14, "O-": 1e14}, max_np_factor=8)


DECKS = {"aro2_33x17": (aro2_deck(33, 17, 0.01, 40), 5), "aro2_65x33": (aro2_deck(65, 33, 0.04, 30), 17),
         "o2_33x17": (o2_deck(33, 17, 0.01, 40), 8), "o2_65x33": (o2_deck(65, 33, 0.04, 30), 9)}
# O2 decks: 0 = the reference's electrons-only launch, 1 = every species collides
ALL = {"o2_33x17": 1, "o2_65x33": 0}


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32 if a.dtype.itemsize == 4 else np.uint64)


def pair(name):
    deck, seed = DECKS[name]
    kw = dict(OPTS, o2_all_species=ALL.get(name, 0))
    S = hpic.Setup(deck, seed=seed, **kw)
    case = hpic.Case(setup=S, seed=seed, **kw)
    o = oracle.Oracle(S.table, S.info, case.opts, 32, pcg_cluster=case.info.pcg_cluster,
                      pcg_block=case.info.pcg_block)
    for s in range(S.info.nsp):
        counts, arrs = S.particles(s, layout=0)
        o.set_particles(s, counts, *arrs)
    o.DepositBasic()
    return case, o


def check(case, o, what):
    for s in range(case.info.nsp):
        gc, ga = case.particles(s)
        oc, oa = o.particles(s)
        assert np.array_equal(gc, oc), f"{what}: species {s} counts differ"
        for k, (a, b) in enumerate(zip(ga, oa)):
            assert np.array_equal(bits(a), bits(b)), f"{what}: species {s} component {k} differs"
    assert np.array_equal(case.grid("MCC_COUNT"), o.counters()[1]), f"{what}: channel tallies differ"


@pytest.mark.parametrize("name", list(DECKS))
def test_aro2_mcc_bit_exact(name):
    case, o = pair(name)
    for t in (1, 2, 3):
        case.set_tstep(t)
        case.MCC()
        o.MCC(t)
        check(case, o, f"after MCC {t}")
    tallies = case.grid("MCC_COUNT").reshape(-1, case.info.mcc_stride).sum(0)
    assert tallies.sum() > 0


@pytest.mark.parametrize("name", list(DECKS))
def test_aro2_steps_bit_exact(name):
    case, o = pair(name)
    n = 30
    case.step(n)
    o.run(0, n, accumulate=True)
    check(case, o, f"after {n} steps")
    for g in ("DEN", "PHI", "EX", "EY"):
        assert np.array_equal(bits(case.grid(g)), bits(o.grid(g))), g
    assert case.status() == 0
    tallies = case.grid("MCC_COUNT").reshape(-1, case.info.mcc_stride).sum(0)
    if name.startswith("aro2"):
        # electron-neutral, ion-neutral and charge-transfer channels all fire
        assert tallies[0] > 0 and tallies[65] + tallies[66] > 0 and tallies[53] > 0
    elif ALL[name]:
        assert tallies[0] > 0 and tallies[47:58].sum() > 0  # ions collide too
    else:
        assert tallies[0] > 0 and tallies[41:58].sum() == 0  # electrons only, as the reference
