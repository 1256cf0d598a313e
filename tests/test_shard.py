"""Independent cases across the GPUs of a node (hpic.shard): the placement
(hp_partition_cases) on CPU, the placement and result gather across two gloo
ranks on CPU (each rank's share run by a stand-in runner), and on one GPU the
sharded run against every case run alone."""
import os
import socket
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(REPO, "hybrid-final_b200"))

import hpic  # noqa: E402
from hpic import shard  # noqa: E402
from hpic.decks import ccp_deck  # noqa: E402


def _decks():
    # slots for 8x the load per cell: no cell reaches the half-full (ReArg) status
    return [ccp_deck(33, 17, 0.01, 0.005, ppc=8, voltage=150.0, max_np_factor=8),
            ccp_deck(65, 33, 0.02, 0.01, ppc=12, voltage=100.0, max_np_factor=8),
            ccp_deck(33, 17, 0.01, 0.005, ppc=16, voltage=200.0, gas="ArO2", pressure_torr=0.1, max_np_factor=8),
            ccp_deck(17, 9, 0.005, 0.0025, ppc=20, voltage=80.0, max_np_factor=8),
            ccp_deck(65, 33, 0.02, 0.01, ppc=6, voltage=250.0, max_np_factor=8)]


def test_longest_first_placement():
    # 5 -> 0, 4 -> 1, 3 -> 1 (4 < 5), 3 -> 0 (5 < 7), 2 -> 1 (7 < 8), 1 -> 0 (8 < 9)
    assert shard.partition([5, 4, 3, 3, 2, 1], [1] * 6, 2) == [0, 1, 1, 0, 1, 0]
    # ties go to the lower case index first and to the lower device
    assert shard.partition([1, 1, 1, 1], [1] * 4, 3) == [0, 1, 2, 0]
    assert shard.partition([], [], 4) == []
    # loads end balanced within the largest weight
    rng = np.random.default_rng(3)
    w = rng.uniform(1, 100, 200)
    place = shard.partition(w, [1] * 200, 8)
    loads = np.bincount(place, weights=w, minlength=8)
    assert loads.max() - loads.min() <= w.max()


def test_budget_limits_the_bytes_per_device():
    w = [10, 9, 8, 7]
    b = [60, 50, 40, 30]
    place = shard.partition(w, b, 2, budget=100)
    used = np.bincount(place, weights=b, minlength=2)
    assert used.max() <= 100
    # the heaviest case would go to device 0, which is full: device 1 instead
    assert shard.partition([10, 9, 1], [90, 5, 20], 2, budget=100) == [0, 1, 1]
    # a case larger than every budget is refused
    with pytest.raises(hpic.HpicError) as e:
        shard.partition([1, 2], [10, 200], 2, budget=100)
    assert e.value.status == hpic.HP_ERR_CAPACITY
    with pytest.raises(hpic.HpicError):
        shard.partition([1, -1], [1, 1], 2)


def test_footprint_from_the_host_setup():
    work, nbytes = shard.footprint(_decks()[1], seed=4)
    assert work == 64 * 32 * 12 * 2  # cells x ppc x species
    big_work, big_bytes = shard.footprint(ccp_deck(129, 65, 0.04, 0.02, ppc=12), seed=4)
    assert big_work == 4 * work and big_bytes > 3 * nbytes > 0


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _fake_runner(items, steps, device, **opts):
    # stands in for the GPU run: a result that names the case and its deck
    return [dict(case=k, steps=steps, grid=(len(deck), seed), device=device) for k, deck, seed in items]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as td
    sys.path.insert(0, os.path.join(REPO, "hybrid-final_b200"))
    from hpic import shard as sh
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    td.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        decks = [hpic.deck_text(d) for d in _decks()]
        res, place = sh.run_sharded(decks, 7, seeds=[11, 12, 13, 14, 15], dist=td, device=rank,
                                    runner=_fake_runner)
        out.put((rank, res, place))
        td.barrier()
    finally:
        td.destroy_process_group()


def test_two_ranks_place_run_and_gather():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted([q.get(timeout=180) for _ in procs], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, res0, place0), (_, res1, place1) = got
    assert place0 == place1  # every rank computes the same placement
    assert res1 is None
    decks = [hpic.deck_text(d) for d in _decks()]
    sizes = [shard.footprint(d, s) for d, s in zip(decks, [11, 12, 13, 14, 15])]
    assert place0 == shard.partition([w for w, _ in sizes], [b for _, b in sizes], 2)
    assert set(place0) == {0, 1}
    assert [r["case"] for r in res0] == list(range(5))
    for k, r in enumerate(res0):
        assert r["rank"] == place0[k] and r["device"] == place0[k]
        assert r["grid"] == (len(decks[k]), 11 + k) and r["steps"] == 7


@pytest.mark.gpu
def test_sharded_run_equals_each_case_alone():
    decks = _decks()
    seeds = [21, 22, 23, 24, 25]
    res, place = shard.run_sharded(decks, 12, seeds=seeds, device=0)
    assert place == [0] * 5
    for k, (deck, seed) in enumerate(zip(decks, seeds)):
        c = hpic.Case(deck=deck, seed=seed)
        c.step(12)
        r = res[k]
        assert r["status"] == c.status() == 0
        assert r["steps"] == 12 and r["pushes"] == c.pushes()
        assert np.array_equal(r["ave_phi"].view(np.uint64), c.grid("AVE_PHI").view(np.uint64))
        assert np.array_equal(r["ave_den"].reshape(-1).view(np.uint64), c.grid("AVE_DEN").view(np.uint64))
        c.close()
