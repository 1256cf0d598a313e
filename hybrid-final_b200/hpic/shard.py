"""Independent cases on the GPUs of one node (the batched form across GPUs).

Cases have no exchange step, so they shard by case: one process per GPU
(torch.distributed, any backend), cases placed on devices by
`hp_partition_cases` (longest-first greedy on the work per step, within each
device's memory budget), each rank running its share as one batch per gas,
and rank 0 gathering the per-case results.  The only collectives are two
exchanges of small host objects: the cases' footprints (each rank sizes a
slice of them) and the results.

    results = run_sharded(decks, steps=2000, seeds=seeds, dist=torch.distributed)

Every rank passes the same arguments; rank 0 gets the list of results in the
order of `decks`, the other ranks get None.
"""
import ctypes as C

import numpy as np

from . import Batch, Case, Setup, _check, lib

_SIG_DONE = False


def _bind():
    global _SIG_DONE
    L = lib()
    if not _SIG_DONE:
        fn = L.hp_partition_cases
        fn.restype = C.c_int
        fn.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_size_t), C.c_int, C.c_int, C.POINTER(C.c_size_t),
                       C.POINTER(C.c_int)]
        _SIG_DONE = True
    return L


def partition(weights, nbytes, ndevices, budget=None):
    """Device index of every case (hp_partition_cases).  budget: bytes per
    device (a number for all, a list per device, or None)."""
    L = _bind()
    n = len(weights)
    w = np.ascontiguousarray(weights, dtype=np.float64)
    b = np.ascontiguousarray(nbytes, dtype=np.uint64)
    out = np.zeros(max(n, 1), dtype=np.int32)
    bud = None
    if budget is not None:
        bud = np.ascontiguousarray(np.broadcast_to(np.asarray(budget, dtype=np.uint64), (ndevices,)))
    st = L.hp_partition_cases(w.ctypes.data_as(C.POINTER(C.c_double)), b.ctypes.data_as(C.POINTER(C.c_size_t)), n,
                              int(ndevices),
                              None if bud is None else bud.ctypes.data_as(C.POINTER(C.c_size_t)),
                              out.ctypes.data_as(C.POINTER(C.c_int)))
    _check(st)
    return out[:n].tolist()


def footprint(deck, seed=1, **case_opts):
    """(work per step, device bytes) of a case, from its host set-up: the
    particles it starts with and hp_case_info.device_bytes."""
    opts = dict(case_opts)
    opts.setdefault("gpu_load", 1)  # sizes only: the particles need not be drawn
    s = Setup(deck, seed=seed, **opts)
    sp = s.table("species").reshape(-1, 16)
    work = float(sp[: s.info.nsp, 13].sum())
    return work, int(s.info.device_bytes)


def run_local(items, steps, device=0, **case_opts):
    """Run cases on this process's GPU: items = [(k, deck, seed)], one batch
    per gas, `steps` steps each.  Returns one dict per case."""
    cases, keys = [], []
    for k, deck, seed in items:
        cases.append(Case(deck=deck, seed=seed, device=device, **case_opts))
        keys.append(k)
    by_gas = {}
    for c in cases:
        by_gas.setdefault(c.info.main_gas, []).append(c)
    batches = [Batch(cs) for cs in by_gas.values()]
    for b in batches:
        b.step(steps)
    out = []
    for k, c in zip(keys, cases):
        out.append(dict(case=k, status=c.status(), steps=int(c.tstep()), pushes=int(c.pushes()),
                        ngx=c.info.ngx, ngy=c.info.ngy, nsp=c.info.nsp,
                        ave_den=c.grid("AVE_DEN").reshape(c.info.nsp, -1), ave_phi=c.grid("AVE_PHI")))
    for b in batches:
        b.close()
    for c in cases:
        c.close()
    return out


def run_sharded(decks, steps, seeds=None, dist=None, budget_bytes=None, device=None, runner=None, sizes=None,
                **case_opts):
    """Shard independent cases over the ranks of `dist` (torch.distributed,
    initialised; None: one process) and gather their results on rank 0.

    decks: the cases (dicts, JSON texts or paths); seeds: one per case
    (default 1, 2, ...); budget_bytes: device memory per GPU for the
    placement; device: this rank's CUDA device (default: the rank's local
    index); runner(items, steps, device, **case_opts): what runs this rank's
    share (default run_local); sizes: [(work, bytes)] per case when known,
    else each rank sizes every world-th case from its host set-up and the
    ranks exchange them.  Returns (results in deck order, placement) on
    rank 0, (None, placement) elsewhere; a result carries the rank that ran
    it."""
    n = len(decks)
    seeds = list(seeds) if seeds is not None else list(range(1, n + 1))
    world = dist.get_world_size() if dist is not None else 1
    rank = dist.get_rank() if dist is not None else 0
    if device is None:
        import os
        device = int(os.environ.get("LOCAL_RANK", rank))
    if sizes is None:
        mine = {k: footprint(decks[k], seeds[k], **case_opts) for k in range(rank, n, world)}
        if dist is not None:
            parts = [None] * world
            dist.all_gather_object(parts, mine)
        else:
            parts = [mine]
        sizes = [None] * n
        for p in parts:
            for k, v in p.items():
                sizes[k] = v
    place = partition([w for w, _ in sizes], [b for _, b in sizes], world, budget_bytes)
    items = [(k, decks[k], seeds[k]) for k in range(n) if place[k] == rank]
    run = runner or run_local
    local = run(items, steps, device, **case_opts) if items else []
    for r in local:
        r["rank"] = rank
    if dist is not None:
        gathered = [None] * world if rank == 0 else None
        dist.gather_object(local, gathered, dst=0)
    else:
        gathered = [local]
    if rank != 0:
        return None, place
    by_case = {}
    for part in gathered:
        for r in part:
            by_case[r["case"]] = r
    return [by_case.get(k) for k in range(n)], place
