"""Bit-exact GPU vs oracle on the benchmark's own configurations, at full size.

The operator tests use decks of at most 65x33 nodes; several code paths only
appear on larger grids (the 16-CTA PCG cluster, the separable solver's GEMM
tiling at 513 columns, cells with 800 slots, far-mover buckets under strong
drive).  Here the library and the oracle run the cases the benchmark quotes:

* the reference's CPU-sized Ar case, 129x65 nodes, 50 particles per cell and
  species, for 50 steps, in field modes 0 (the reference's PCG rule) and 2;
* the precision-form Ar case, 513x257 nodes, 200 particles per cell and
  species (52M particles), for 3 steps, and its field solve in modes 1 and 2;
* the 80/20 Ar/O2 case, 257x129 nodes, 100 particles per cell, for 5 steps.

Everything is compared bit for bit, as in test_gpu_ops.py."""
import os
import sys

import numpy as np
import pytest

import hpic
import oracle

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from bench import WORKLOADS, make_deck  # noqa: E402

pytestmark = pytest.mark.gpu


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32 if a.dtype.itemsize == 4 else np.uint64)


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and np.array_equal(bits(a), bits(b))


def pair(workload, seed=1000, **opts):
    deck = make_deck(WORKLOADS[workload])
    kw = dict(seed=seed, gas_temp_mode=1, **opts)
    S = hpic.Setup(deck, **kw)
    case = hpic.Case(setup=S, **kw)
    info = case.info
    o = oracle.Oracle(S.table, S.info, case.opts, 32, pcg_cluster=info.pcg_cluster, pcg_block=info.pcg_block)
    for s in range(S.info.nsp):
        counts, arrs = S.particles(s, layout=0)
        o.set_particles(s, counts, *arrs)
    o.DepositBasic()
    del S
    return case, o


def check_state(case, o, what):
    for s in range(case.info.nsp):
        gc, ga = case.particles(s)
        oc, oa = o.particles(s)
        assert np.array_equal(gc, oc), f"{what} species {s}: counts differ"
        for k, (a, b) in enumerate(zip(ga, oa)):
            assert same(a, b), f"{what} species {s}: component {k} differs"
    for g in ("DEN", "SOURCE", "PHI", "EX", "EY"):
        assert same(case.grid(g), o.grid(g)), f"{what}: {g} differs"
    assert np.array_equal(case.grid("MCC_COUNT"), o.counters()[1]), f"{what}: collision tallies differ"
    assert case.status() == 0


@pytest.mark.parametrize("field_mode,move_mode", [(0, 0), (2, 1)])
def test_ar_129x65_50ppc_50_steps(field_mode, move_mode):
    case, o = pair("ar_129x65_50ppc", field_mode=field_mode, move_mode=move_mode)
    case.step(50)
    o.run(0, 50, accumulate=True)
    check_state(case, o, f"129x65, field_mode {field_mode}, move_mode {move_mode}, 50 steps")
    d, p, n = o.averages()
    assert same(case.grid("AVE_DEN"), d) and same(case.grid("AVE_PHI"), p) and n == 50


def test_ar_513x257_200ppc_3_steps():
    case, o = pair("ar_513x257_200ppc", field_mode=2, move_mode=1)
    assert case.info.cap[0] >= 800
    case.step(3)
    o.run(0, 3, accumulate=True)
    check_state(case, o, "513x257, 3 steps")


@pytest.mark.parametrize("field_mode", [0, 1, 2])
def test_ar_513x257_field(field_mode):
    """The field solve of the 513x257 case on its initial charge: the
    whole-GPU cooperative PCG (131k nodes, above one 16-CTA cluster) with the
    reference's rule (mode 0) and with FP64 refinement (mode 1), and the
    separable solver (mode 2)."""
    case, o = pair("ar_513x257_200ppc", field_mode=field_mode, move_mode=1)
    if field_mode in (0, 1):
        assert case.info.pcg_cluster == (513 * 257 + 1023) // 1024  # one CTA per 1024 nodes
    case.set_tstep(1)
    case.Field()
    o.Field(1)
    for g in ("PHI_POIS", "PHI", "EX", "EY"):
        assert same(case.grid(g), o.grid(g)), g
    assert case.pcg_iters()[0] == o.counters()[2][0]
    assert case.status() == 0


def test_aro2_257x129_100ppc_5_steps():
    case, o = pair("aro2_257x129_100ppc", field_mode=2, move_mode=1)
    assert case.info.nsp == 5
    case.step(5)
    o.run(0, 5, accumulate=True)
    check_state(case, o, "Ar/O2 257x129, 5 steps")


@pytest.mark.parametrize("field_mode", [0, 1])
def test_whole_gpu_pcg_through_the_step_graph(field_mode):
    """A 321x225 case (72k nodes) solves with the cooperative whole-GPU PCG
    (71 CTAs) inside the captured step graph, three steps, and in a batch
    next to a cluster-solved case: bit for bit with the oracle."""
    from hpic.decks import ccp_deck
    deck = ccp_deck(321, 225, 0.1, 0.07, ppc=4, voltage=150.0, max_np_factor=16)
    kw = dict(seed=77, gas_temp_mode=1, field_mode=field_mode, move_mode=1)
    S = hpic.Setup(deck, **kw)
    case = hpic.Case(setup=S, **kw)
    assert case.info.pcg_cluster == (321 * 225 + 1023) // 1024
    o = oracle.Oracle(S.table, S.info, case.opts, 32, pcg_cluster=case.info.pcg_cluster,
                      pcg_block=case.info.pcg_block)
    for s in range(S.info.nsp):
        counts, arrs = S.particles(s, layout=0)
        o.set_particles(s, counts, *arrs)
    o.DepositBasic()
    small = hpic.Case(deck=ccp_deck(65, 33, 0.02, 0.01, ppc=8), seed=5, field_mode=field_mode)
    batch = hpic.Batch([small, case])
    batch.step(3)
    batch.close()
    o.run(0, 3)
    check_state(case, o, "321x225 grid PCG, 3 steps")
    assert case.pcg_iters()[0] == o.counters()[2][0]
