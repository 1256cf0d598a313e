"""The fluid species on the GPU against the oracle, bit for bit.

The decks set AverageIter to 3, so the cycle averages at steps 4, 8, 12, ...
and the continuity solve runs from step 5 on: within 16 steps every phase of
the cycle runs several times (the electron density sum, the averaged
collision rates, the sources of every fluid species, the node copy that the
collisions read, the Ar collision probability that follows the Ar* density,
and the x and y line sweeps).  The oracle's continuity solve is pinned to the
reference's own code in test_fluid.py."""
import copy

import numpy as np
import pytest

import hpic
import oracle
from hpic.decks import block_deck, ccp_deck

pytestmark = pytest.mark.gpu

FLUID = ("FLUID_CELL_DEN", "FLUID_DEN", "FLUID_SOURCE", "FLUID_FLUX_X", "FLUID_FLUX_Y")


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32 if a.dtype.itemsize == 4 else np.uint64)


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and np.array_equal(bits(a), bits(b))


# initial fluid densities (m^-3); the deck builder leaves them 0
FLUID_DENSITY = {"Ar*": 1e16, "O2A": 1e17, "O2B": 1e16, "OP": 1e18, "OD": 1e15}


def fluid_deck(deck, average_iter=3):
    """The deck with AverageIter set and the fluid species loaded."""
    d = copy.deepcopy(deck)

    def walk(o):
        if isinstance(o, dict):
            for k, v in o.items():
                if k == "AverageIter":
                    o[k] = average_iter
                elif k in FLUID_DENSITY and isinstance(v, dict) and "Density" in v:
                    v["Density"] = FLUID_DENSITY[k]
                else:
                    walk(v)
        elif isinstance(o, list):
            for v in o:
                walk(v)

    walk(d)
    return d


DECKS = {
    "ar_33x17": (fluid_deck(ccp_deck(33, 17, 0.01, 0.005, ppc=20, pressure_torr=0.1, voltage=200.0)), 777),
    "ar_block_33x21": (fluid_deck(block_deck()), 4242),
    "o2_33x17": (fluid_deck(ccp_deck(33, 17, 0.01, 0.005, gas="O2", ppc=12, pressure_torr=0.1, voltage=200.0,
                                     te_ev=3.0, ion_density={"O2+": 1e15, "O+": 1e14, "O-": 1e14})), 616),
    "aro2_33x17": (fluid_deck(ccp_deck(33, 17, 0.01, 0.005, gas="ArO2", ppc=12, pressure_torr=0.1, voltage=200.0,
                                       te_ev=3.0, ion_density={"Ar+": 1e15, "O2+": 2e14, "O+": 0.0, "O-": 2e14})),
                   515),
}
CAP = {"ar_block_33x21": 256}


def pair(name, **extra):
    deck, seed = DECKS[name]
    kw = dict(seed=seed, field_mode=0, move_mode=0, cap_per_cell=CAP.get(name, 0), **extra)
    S = hpic.Setup(deck, **kw)
    case = hpic.Case(setup=S, **kw)
    info = case.info
    o = oracle.Oracle(S.table, S.info, case.opts, 32, pcg_cluster=info.pcg_cluster, pcg_block=info.pcg_block)
    for s in range(S.info.nsp):
        counts, arrs = S.particles(s, layout=0)
        o.set_particles(s, counts, *arrs)
    o.DepositBasic()
    return case, o, S


def check(case, o, what):
    for s in range(case.info.nsp):
        gc, ga = case.particles(s)
        oc, oa = o.particles(s)
        assert np.array_equal(gc, oc), f"{what} species {s}: counts differ"
        for k, (a, b) in enumerate(zip(ga, oa)):
            assert same(a, b), f"{what} species {s}: component {k} differs"
    for g in ("DEN", "PHI", "EX", "EY") + FLUID:
        assert same(case.grid(g), o.grid(g)), f"{what}: {g} differs"
    assert np.array_equal(case.grid("MCC_COUNT"), o.counters()[1]), f"{what}: collision tallies differ"
    assert case.status() == 0


@pytest.mark.parametrize("name", list(DECKS))
def test_fluid_cycle_bit_exact(name):
    case, o, S = pair(name)
    assert case.info.n_fluid >= 1
    for k in range(4):
        case.step(4)
        o.run(4 * k, 4, accumulate=True)
        check(case, o, f"{name}, step {4 * (k + 1)}")
    # the cycle did run: sources were set and the densities moved
    assert np.any(case.grid("FLUID_SOURCE") != 0)
    assert not same(case.grid("FLUID_CELL_DEN"), S.table("fluid_cell_den"))


def test_fluid_fixed_holds_the_initial_densities():
    case, o, S = pair("ar_33x17", fluid_fixed=1)
    case.step(12)
    o.run(0, 12, accumulate=True)
    check(case, o, "fluid_fixed")
    assert same(case.grid("FLUID_CELL_DEN"), S.table("fluid_cell_den"))
    assert same(case.grid("FLUID_DEN"), S.table("fluid_den"))
    assert not np.any(case.grid("FLUID_SOURCE"))


def test_fluid_in_a_batch_equals_alone():
    """Cases with different line sets and species counts in one batch (one
    launch per phase) give what each gives alone."""
    names = ["ar_33x17", "ar_block_33x21"]
    alone = []
    for n in names:
        case, _, _ = pair(n)
        case.step(10)
        alone.append({g: case.grid(g) for g in FLUID + ("DEN",)})
    cases = [pair(n)[0] for n in names]
    b = hpic.Batch(cases)
    b.step(10)
    for n, c, ref in zip(names, cases, alone):
        for g, v in ref.items():
            assert same(c.grid(g), v), f"{n}: {g} differs in the batch"


def test_fluid_state_survives_a_checkpoint(tmp_path):
    """A checkpoint in the middle of an averaging window resumes bit for bit."""
    case, _, _ = pair("ar_33x17")
    case.step(6)
    path = str(tmp_path / "ck.bin")
    case.save(path)
    case.step(6)
    ref = {g: case.grid(g) for g in FLUID + ("DEN",)}
    other, _, _ = pair("ar_33x17")
    other.load(path)
    other.step(6)
    for g, v in ref.items():
        assert same(other.grid(g), v), g
