"""GPU operators vs. the CPU oracle, through the C ABI.

The oracle evaluates the same single-precision arithmetic in the same order
(including the warp and cluster reduction trees), so every operator is
compared bit for bit: positions, velocities, cell counts, mover codes,
collision channels, created particles, densities, potentials and fields.
"""
import numpy as np
import pytest

import hpic
import oracle
from hpic.decks import block_deck, ccp_deck, dielectric_deck

pytestmark = pytest.mark.gpu


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32 if a.dtype.itemsize == 4 else np.uint64)


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and np.array_equal(bits(a), bits(b))


DECKS = {
    "ar_17x9": (ccp_deck(17, 9, 0.005, 0.0025, ppc=10), 12345),
    "ar_33x17_hv": (ccp_deck(33, 17, 0.01, 0.005, ppc=20, pressure_torr=0.1, voltage=300.0), 777),
    "ar_65x33": (ccp_deck(65, 33, 0.02, 0.01, ppc=30), 99),
    "ar_block_33x21": (block_deck(), 4242),
    # two 1-2-1 density smoothing passes per Deposit (Smooth_121_x/_y)
    "ar_33x17_smooth2": (ccp_deck(33, 17, 0.01, 0.005, ppc=20, pressure_torr=0.1, voltage=300.0, smoothing=2), 778),
    # a dielectric slab on the driven electrode and a dielectric block inside
    "ar_diel_33x21": (dielectric_deck(), 4343),
    # a power-driven source (0.5 W), its amplitude revised every 20 steps
    "ar_33x17_power": (ccp_deck(33, 17, 0.01, 0.005, ppc=20, power_w=0.5, pd_interval=0.05), 55),
}
# slots per cell where the deck's Max_np / Gsize leaves too little room for
# the charge that gathers in front of the floating block
CAP = {"ar_block_33x21": 256, "ar_diel_33x21": 256}


def pair(name, field_mode=0, move_mode=0, **extra):
    deck, seed = DECKS[name]
    kw = dict(seed=seed, field_mode=field_mode, move_mode=move_mode, cap_per_cell=CAP.get(name, 0), **extra)
    S = hpic.Setup(deck, **kw)
    case = hpic.Case(setup=S, **kw)
    info = case.info
    o = oracle.Oracle(S.table, S.info, case.opts, 32, pcg_cluster=info.pcg_cluster, pcg_block=info.pcg_block)
    for s in range(S.info.nsp):
        counts, arrs = S.particles(s, layout=0)
        o.set_particles(s, counts, *arrs)
    o.DepositBasic()  # the library's initial Deposit_Basic
    return case, o


def check_particles(case, o, what=""):
    for s in range(case.info.nsp):
        gc, ga = case.particles(s)
        oc, oa = o.particles(s)
        assert np.array_equal(gc, oc), f"{what} species {s}: counts differ"
        for k, (a, b) in enumerate(zip(ga, oa)):
            assert same(a, b), f"{what} species {s}: component {k} differs"


def check_surface(case, o, what=""):
    """Dielectric surface weights and Sigma, where the deck has dielectrics."""
    if not case.info.n_dielectric:
        return
    assert np.array_equal(case.grid("SURFACE_CHARGE"), o.grid("SURFACE_CHARGE")), f"{what}: surface charge differs"
    assert same(case.grid("SIGMA"), o.grid("SIGMA")), f"{what}: Sigma differs"


def check_grids(case, o, names=("DEN", "SOURCE"), what=""):
    for n in names:
        g = case.grid(n)
        r = o.grid(n)
        assert same(g, r), f"{what}: grid {n} differs (max |d| {np.abs(g.astype(np.float64) - r).max()})"


@pytest.mark.parametrize("name", list(DECKS))
def test_initial_deposit(name):
    case, o = pair(name)
    check_grids(case, o, ("DEN", "SOURCE"), "initial deposit")
    g = case.grid("PCG_B")
    assert same(g, o.grid("B"))


@pytest.mark.parametrize("name", list(DECKS))
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_field(name, mode):
    case, o = pair(name, field_mode=mode)
    case.set_tstep(1)
    case.Field()
    o.Field(1)
    for n in ("PHI_POIS", "PHI", "EX", "EY"):
        assert same(case.grid(n), o.grid(n)), n
    assert case.pcg_iters()[0] == o.counters()[2][0]
    assert case.status() == 0


@pytest.mark.parametrize("name", list(DECKS))
@pytest.mark.parametrize("move_mode", [0, 1])
def test_move_and_sort(name, move_mode):
    case, o = pair(name, move_mode=move_mode)
    case.set_tstep(1)
    case.Field()
    o.Field(1)
    case.Move()
    o.Move()
    check_particles(case, o, "after Move (stayers)")
    for s in range(case.info.nsp):
        gc, ga, gcode = case.movers(s)
        oc, oa, ocode = o.movers(s)
        assert np.array_equal(gc, oc)
        assert np.array_equal(gcode, ocode)
        for a, b in zip(ga, oa):
            assert same(a, b)
    case.SortBoundary()
    o.SortBoundary()
    check_particles(case, o, "after SortBoundary")
    assert same(case.grid("COND_CHARGE"), o.counters()[0][: case.info.nsp * case.info.cond_numr])
    check_surface(case, o, "after SortBoundary")


@pytest.mark.parametrize("name", list(DECKS))
@pytest.mark.parametrize("group", [1, 2, 4, 8, 16])
def test_mcc(name, group):
    """Ar MCC with 1-16 consecutive cells per warp sharing collision batches."""
    case, o = pair(name)
    case.set_tune(mcc_cells_per_warp=group)
    for t in (1, 2, 3):
        case.set_tstep(t)
        case.MCC()
        o.MCC(t)
        check_particles(case, o, f"after MCC step {t}")
    assert np.array_equal(case.grid("MCC_COUNT"), o.counters()[1])
    assert case.grid("MCC_COUNT").reshape(-1, 8).sum() > 0


@pytest.mark.parametrize("name", list(DECKS))
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_steps_bit_exact(name, mode):
    case, o = pair(name, field_mode=mode)
    n = 25
    case.step(n)
    o.run(0, n, accumulate=True)
    check_particles(case, o, f"after {n} steps")
    check_grids(case, o, ("DEN", "SOURCE"), "after steps")
    check_surface(case, o, f"after {n} steps")
    for g in ("PHI", "EX", "EY"):
        assert same(case.grid(g), o.grid(g)), g
    assert np.array_equal(case.grid("MCC_COUNT"), o.counters()[1])
    d, p, cnt = o.averages()
    assert case.average_count() == cnt == n
    assert same(case.grid("AVE_DEN"), d)
    assert same(case.grid("AVE_PHI"), p)
    src, ex, ey = o.field_averages()
    assert same(case.grid("AVE_SOURCE"), src)
    assert same(case.grid("AVE_EX"), ex)
    assert same(case.grid("AVE_EY"), ey)
    assert case.status() == 0
    assert case.tstep() == n


@pytest.mark.parametrize("name", list(DECKS))
@pytest.mark.parametrize("ppl", [1, 2, 4])
def test_walk_steps_bit_exact(name, ppl):
    """move_mode 1 (cell-by-cell walk) with the separable field solve; Move
    with one or four particles per lane."""
    case, o = pair(name, field_mode=2, move_mode=1)
    case.set_tune(move_unroll=ppl)
    n = 25
    case.step(n)
    o.run(0, n, accumulate=True)
    check_particles(case, o, f"after {n} steps")
    check_grids(case, o, ("DEN", "SOURCE"), "after steps")
    check_surface(case, o, f"after {n} walk steps")
    assert same(case.grid("COND_CHARGE"), o.counters()[0][: case.info.nsp * case.info.cond_numr])
    assert case.status() == 0


@pytest.mark.parametrize("name", ["ar_33x17_hv", "ar_block_33x21"])
def test_eedf_counts(name):
    """The electron energy histogram (every 5th step) counts the same
    electrons into the same 0.25 eV bins as the oracle."""
    case, o = pair(name, field_mode=2, move_mode=1, eedf_every=5)
    n = 23
    case.step(n)
    o.run(0, n, accumulate=True)
    h = case.grid("EEDF")
    assert h.dtype == np.uint64 and h.size == hpic.EEDF_BINS + 1
    assert np.array_equal(h, o.eedf())
    # four samples (steps 5, 10, 15, 20) of every electron present then
    assert 0 < int(h.sum()) <= 4 * case.info.cap[0] * case.info.Csize
    case.reset_averages()
    assert int(case.grid("EEDF").sum()) == 0


def fast_electrons(case, o, cells_per_step, every=3):
    """Give every `every`-th electron a velocity of `cells_per_step` cells per
    step in x and half that in y (signs alternating), on both sides."""
    info = case.info
    counts, (x, y, vx, vy, vz) = case.particles(0)
    vcx = np.float32(cells_per_step * info.dx / info.dt)
    vcy = np.float32(0.5 * cells_per_step * info.dy / info.dt)
    k = np.arange(x.size)
    sel = k % every == 0
    sign = np.where((k // every) % 2 == 0, 1, -1).astype(np.float32)
    vx = np.where(sel, sign * vcx, vx).astype(np.float32)
    vy = np.where(sel, -sign * vcy, vy).astype(np.float32)
    case.set_particles(0, counts, x, y, vx, vy, vz)
    o.set_particles(0, counts, x, y, vx, vy, vz)


@pytest.mark.parametrize("cells", [2.6, 7.3])
@pytest.mark.parametrize("ppl", [1, 2, 4])
def test_far_movers_bit_exact(cells, ppl):
    """Electrons crossing several cells per push: the walk, the reflections on
    the side walls, absorption at the electrodes and the far-mover order."""
    case, o = pair("ar_65x33", field_mode=2, move_mode=1)
    case.set_tune(move_unroll=ppl)
    fast_electrons(case, o, cells)
    for t in (1, 2):
        case.set_tstep(t)
        case.Field()
        o.Field(t)
        case.Move()
        o.Move()
        gc, ga, gcode = case.movers(0)
        oc, oa, ocode = o.movers(0)
        assert np.array_equal(gc, oc) and np.array_equal(gcode, ocode)
        assert (gcode == 14).sum() > 0, "no mover went beyond the 3x3 neighbourhood"
        for a, b in zip(ga, oa):
            assert same(a, b)
        case.SortBoundary()
        o.SortBoundary()
        check_particles(case, o, f"after walk sort {t}")
        assert same(case.grid("COND_CHARGE"), o.counters()[0][: case.info.nsp * case.info.cond_numr])
    _, (x, y, *_rest) = case.particles(0)
    assert x.min() >= 0 and x.max() < 1 and y.min() >= 0 and y.max() < 1
    assert case.status() == 0


def test_reference_wrap_leaves_offsets_outside_the_cell():
    """move_mode 0 keeps the reference's single wrap: a particle faster than a
    cell per push ends with an offset outside [0, 1)."""
    case, o = pair("ar_65x33", field_mode=2, move_mode=0)
    fast_electrons(case, o, 2.6)
    case.set_tstep(1)
    case.Field()
    case.Move()
    case.SortBoundary()
    _, (x, *_rest) = case.particles(0)
    assert x.max() >= 1 or x.min() < 0


def test_walk_stays_finite_over_many_rf_periods_fraction():
    """At the decks' dt (1/400 of the RF period) the reference wrap lets
    offsets grow without bound within ~100 steps; the walk keeps every offset
    in [0, 1) and the status clean over 400 steps (one RF period)."""
    deck = ccp_deck(65, 33, 0.02, 0.01, ppc=30)
    case = hpic.Case(deck, seed=5, field_mode=2, move_mode=1, gas_temp_mode=1)
    case.step(400)
    assert case.status() == 0
    for s in range(case.info.nsp):
        _, (x, y, vx, vy, vz) = case.particles(s)
        assert x.size > 1000, f"species {s} nearly gone"
        assert x.min() >= 0 and x.max() < 1 and y.min() >= 0 and y.max() < 1
        assert np.isfinite(vx).all() and np.isfinite(vy).all() and np.isfinite(vz).all()
    assert np.isfinite(case.grid("PHI")).all()


def test_separable_solver_reaches_tolerance():
    """field_mode 2 reaches the FP64 target: ||b - A x|| <= 1e-8 ||b|| (checked
    here in FP64 on the exported operator) and agrees with mode 1."""
    deck, seed = DECKS["ar_65x33"]
    a = hpic.Case(deck, seed=seed, field_mode=2)
    b = hpic.Case(deck, seed=seed, field_mode=1)
    assert a.info.field_mode == 2 and b.info.field_mode == 1
    for c in (a, b):
        c.set_tstep(1)
        c.Field()
    x = a.grid("PCG_X")
    rhs = a.grid("PCG_B")
    st = a.table("stencil").reshape(-1, 5)
    unk = a.table("unk_node")
    ngy = a.info.ngy
    ax = np.zeros(len(unk))
    for k, off in enumerate((-ngy, -1, 0, 1, ngy)):
        nb = np.clip(unk + off, 0, a.info.Gsize - 1)
        ax += np.where(st[:, k] != 0, st[:, k].astype(np.float64) * x[nb], 0.0)
    r = rhs[unk] - ax
    assert np.linalg.norm(r) <= 1e-8 * np.linalg.norm(rhs[unk])
    pa, pb = a.grid("PHI_POIS"), b.grid("PHI_POIS")
    assert np.abs(pa - pb).max() <= 1e-6 * np.abs(pb).max()
    assert a.status() == 0


def test_non_separable_geometry_falls_back():
    """A floating conductor inside the gap breaks the Kronecker structure:
    field_mode 2 must fall back to the PCG refinement and still be exact."""
    import json
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "setup_ar_block_33x21.npz"))
    deck = json.loads(str(g["deck"]))
    c = hpic.Case(deck, seed=5, field_mode=2)
    assert c.info.field_mode == 1
    c.step(3)
    assert c.status() == 0


def test_slot_changes_count_the_shifted_particles():
    """Move counts the particles whose slot changed (movers, and stayers
    compacted below a mover): at most the particles pushed, and every
    mover is one."""
    case, o = pair("ar_65x33", field_mode=2, move_mode=1)
    p0, s0 = case.pushes(), case.slot_changes()
    case.set_tstep(1)
    case.Field()
    case.Move()
    pushed, changed = case.pushes() - p0, case.slot_changes() - s0
    movers = sum(int(case.movers(s)[0].sum()) for s in range(case.info.nsp))
    assert 0 < movers <= changed <= pushed


def test_graph_replay_matches_operator_calls():
    deck, seed = DECKS["ar_33x17_hv"]
    a = hpic.Case(deck, seed=seed)
    b = hpic.Case(deck, seed=seed)
    a.step(6)
    for t in range(1, 7):
        b.set_tstep(t)
        b.Field(); b.Move(); b.SortBoundary(); b.MCC(); b.Deposit()
    for s in range(2):
        ca, pa = a.particles(s)
        cb, pb = b.particles(s)
        assert np.array_equal(ca, cb)
        for x, y in zip(pa, pb):
            assert same(x, y)


@pytest.mark.parametrize("group", [1, 16])
def test_batch_equals_alone(group):
    """A case advanced inside a batch gives the same bits as alone, also when
    MCC cell groups straddle two cases (the 19x10 deck has 162 cells)."""
    decks = [(ccp_deck(19, 10, 0.005625, 0.0028125, ppc=12), 31), DECKS["ar_17x9"], DECKS["ar_33x17_hv"],
             DECKS["ar_65x33"]]
    alone = []
    for deck, seed in decks:
        c = hpic.Case(deck, seed=seed)
        c.step(10)
        alone.append(c)
    mixed = [hpic.Case(deck, seed=seed) for deck, seed in decks]
    b = hpic.Batch(mixed)
    b.set_tune(mcc_cells_per_warp=group)
    b.step(10)
    b.close()
    for a, m in zip(alone, mixed):
        for s in range(2):
            ca, pa = a.particles(s)
            cm, pm = m.particles(s)
            assert np.array_equal(ca, cm)
            for x, y in zip(pa, pm):
                assert same(x, y)
        assert same(a.grid("PHI"), m.grid("PHI"))


def test_rng_matches_curand_philox(tmp_path):
    """hp_rng.h's Philox4x32-10 against curand's (device API) on the same key
    and counter (tests/philox_check.cu)."""
    import os
    import subprocess
    here = os.path.dirname(os.path.abspath(__file__))
    exe = str(tmp_path / "philox_check")
    subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-I",
                    os.path.join(here, "..", "include"), os.path.join(here, "philox_check.cu"), "-o", exe],
                   check=True)
    out = subprocess.run([exe], capture_output=True, text=True).stdout
    assert "mismatches 0 host-vs-device 0" in out, out


def test_dielectric_crossings_bit_exact():
    """Hand-placed electrons entering the dielectric slab and block in every
    direction (E = 0): the surface weights after SortBoundary, then the
    source and Sigma after Deposit, against the oracle."""
    from test_dielectric import place

    case, o = pair("ar_diel_33x21")
    info = case.info
    for s in range(info.nsp):
        z = np.zeros(0, np.float32)
        zc = np.zeros(info.Csize, np.int32)
        case.set_particles(s, zc, z, z, z, z, z)
        o.set_particles(s, zc, z, z, z, z, z)
    S = hpic.Setup(DECKS["ar_diel_33x21"][0], seed=4343, cap_per_cell=CAP["ar_diel_33x21"])
    place(S, o)
    counts, arrs = o.particles(0)
    case.set_particles(0, counts, *arrs)
    case.set_grid("EX", np.zeros(info.Gsize, np.float32))
    case.set_grid("EY", np.zeros(info.Gsize, np.float32))
    case.Move()
    o.Move()
    gc, _, gcode = case.movers(0)
    assert np.all(gcode == 15) and gcode.size > 10
    case.SortBoundary()
    o.SortBoundary()
    sig = case.grid("SURFACE_CHARGE")
    assert np.array_equal(sig, o.grid("SURFACE_CHARGE")) and sig.sum() > 0
    case.Deposit()
    o.Deposit()
    check_grids(case, o, ("DEN", "SOURCE"), "after Deposit")
    check_surface(case, o, "after Deposit")
    assert case.status() == 0


def test_far_bucket_beyond_one_warp():
    """Every electron moved three cells in x at E = 0: each destination
    cell receives a whole source cell's electrons (about 50, more than one
    warp of keys), placed in (source cell, rank) order as the oracle does."""
    deck = ccp_deck(33, 17, 0.01, 0.005, ppc=50)
    S = hpic.Setup(deck, seed=31, field_mode=2, move_mode=1)
    case = hpic.Case(setup=S, seed=31, field_mode=2, move_mode=1)
    info = case.info
    o = oracle.Oracle(S.table, S.info, case.opts, 32, pcg_cluster=info.pcg_cluster, pcg_block=info.pcg_block)
    for s in range(info.nsp):
        counts, arrs = S.particles(s, layout=0)
        o.set_particles(s, counts, *arrs)
    counts, (x, y, vx, vy, vz) = case.particles(0)
    vx = np.full_like(vx, np.float32(3.0 * info.dx / info.dt))
    vy = np.zeros_like(vy)
    case.set_particles(0, counts, x, y, vx, vy, vz)
    o.set_particles(0, counts, x, y, vx, vy, vz)
    for g in ("EX", "EY"):
        z = np.zeros(info.Gsize, np.float32)
        case.set_grid(g, z)
        o.set_grid(g, z)
    case.Move()
    o.Move()
    assert o.far_max() > 32
    case.SortBoundary()
    o.SortBoundary()
    check_particles(case, o, "after a sort with full far buckets")
    assert case.status() == 0


@pytest.mark.parametrize("mode", [1, 2])
def test_power_controller_bit_exact(mode):
    """A power-driven source over 65 steps (revisions at steps 20, 40, 60;
    the first arms the controller): amplitudes, particles and fields as the
    oracle's."""
    case, o = pair("ar_33x17_power", field_mode=mode, move_mode=1)
    assert case.info.power_driven == 1
    a0 = case.grid("SOURCE_AC").copy()
    n = 65
    case.step(n)
    o.run(0, n, accumulate=True)
    amp = case.grid("SOURCE_AC")
    assert same(amp, o.grid("SOURCE_AC")[: amp.size])
    assert amp[0] != a0[0], "the controller revised nothing"
    check_particles(case, o, f"after {n} power-driven steps")
    for g in ("PHI", "EX", "EY"):
        assert same(case.grid(g), o.grid(g)), g
    assert same(case.grid("SIGMA"), o.grid("SIGMA"))
    assert case.status() == 0


def test_mcc_rates_since_reset():
    """hp_get_mcc_rates: the collisions tallied since hp_reset_averages per
    cell and channel, at the cell's lower-left node, times Denscale / (steps
    x dt) in float as the reference's Average_Argon_MCC_rate."""
    case, _ = pair("ar_33x17_hv", field_mode=2, move_mode=1)
    info = case.info
    case.step(10)
    c0 = case.grid("MCC_COUNT").reshape(info.Csize, info.mcc_stride).astype(np.int64)
    case.reset_averages()
    case.step(15)
    c1 = case.grid("MCC_COUNT").reshape(info.Csize, info.mcc_stride).astype(np.int64)
    r = case.mcc_rates()
    assert r.shape == (info.Gsize, info.n_reactions)
    S = hpic.Setup(DECKS["ar_33x17_hv"][0], seed=DECKS["ar_33x17_hv"][1])
    denscale = np.float32(S.table("species").reshape(-1, 16)[0, 8])
    dt = np.float32(S.table("scalars")[0])
    temp = denscale / np.float32(15) / dt
    want = np.zeros_like(r)
    cells = np.arange(info.Csize)
    nodes = (cells // info.ncy) * info.ngy + cells % info.ncy
    for k in range(7):
        want[nodes, k] = temp * (c1 - c0)[:, k].astype(np.float32)
    assert np.array_equal(r, want)
    assert r.sum() > 0


def test_batch_with_dielectric_and_power_cases_equals_alone():
    """Dielectric and power-driven cases inside a batch with a plain one:
    each ends with the same bits as alone (the Sort-phase surface pass and
    the power controller run one block per case of the batch)."""
    decks = [DECKS["ar_diel_33x21"], DECKS["ar_33x17_power"], DECKS["ar_17x9"]]
    kw = [dict(cap_per_cell=CAP["ar_diel_33x21"]), {}, {}]
    opts = dict(field_mode=1, move_mode=1)
    n = 45  # power revisions at steps 20 and 40
    alone = []
    for (deck, seed), k in zip(decks, kw):
        c = hpic.Case(deck, seed=seed, **opts, **k)
        c.step(n)
        alone.append(c)
    mixed = [hpic.Case(deck, seed=seed, **opts, **k) for (deck, seed), k in zip(decks, kw)]
    b = hpic.Batch(mixed)
    b.step(n)
    b.close()
    for a, m in zip(alone, mixed):
        for s in range(a.info.nsp):
            ca, pa = a.particles(s)
            cm, pm = m.particles(s)
            assert np.array_equal(ca, cm)
            for x, y in zip(pa, pm):
                assert same(x, y)
        for g in ("PHI", "SURFACE_CHARGE", "SIGMA", "SOURCE_AC"):
            assert np.array_equal(a.grid(g).view(np.uint8), m.grid(g).view(np.uint8)), g
        assert a.status() == m.status() == 0
    assert alone[0].grid("SURFACE_CHARGE").sum() > 0
    assert alone[1].grid("SOURCE_AC")[0] != np.float32(100.0)
