"""Dielectric blocks: surface charge (SortBoundary's dielectric branch,
src/cuda_Sortboundary.cu:93-207) and its source term (SumSource,
src/cuda_Deposit.cu:35-104), on the oracle.

Particles are placed by hand next to the dielectric slab and block of
hpic.decks.dielectric_deck with E = 0, so that each one enters a dielectric
cell in a known direction; the weights the oracle leaves on the nodes are
compared with a numpy statement of the reference's split, and the source with
the reference's sum.  The GPU kernels are checked against the oracle bit for
bit in test_gpu_ops (deck ar_diel_33x21)."""
import numpy as np

import hpic
import oracle
from hpic.decks import dielectric_deck

F = np.float32
FRAC = float(1 << hpic.SIGMA_FRAC_BITS)

# (cell i, j, direction (di, dj), offset x, y, displacement in cells dx, dy)
CROSSINGS = [
    (5, 3, (0, -1), 0.5, 0.3, 0.25, -0.6),    # down into the slab
    (11, 10, (1, 0), 0.7, 0.4, 0.5, 0.2),     # right into the block
    (11, 10, (1, 0), 0.6, 0.9, 0.55, -0.3),
    (18, 10, (-1, 0), 0.2, 0.5, -0.45, 0.1),  # left into the block
    (14, 12, (0, -1), 0.3, 0.2, 0.1, -0.5),   # down onto the block's top
    (14, 8, (0, 1), 0.6, 0.8, -0.2, 0.5),     # up into the block's bottom
    (11, 12, (1, -1), 0.8, 0.1, 0.5, -0.3),   # diagonals into the block's corners
    (11, 12, (1, -1), 0.9, 0.3, 0.4, -0.5),
    (11, 8, (1, 1), 0.8, 0.9, 0.4, 0.3),
    (11, 8, (1, 1), 0.9, 0.7, 0.3, 0.5),
    (18, 8, (-1, 1), 0.1, 0.9, -0.4, 0.3),
    (18, 12, (-1, -1), 0.2, 0.1, -0.5, -0.3),
    (7, 3, (-1, -1), 0.1, 0.2, -0.4, -0.5),   # diagonal into the slab: the cell below is dielectric
    (7, 3, (1, -1), 0.8, 0.1, 0.5, -0.3),
    (0, 3, (-1, -1), 0.1, 0.1, -0.3, -0.4),   # into the left ghost column: a node off the grid
]


def share(dirn, i, j, x, y, vx, vy, SI, ngy, SY):
    """The reference's split (src/cuda_Sortboundary.cu:93-207) in float32:
    [(node, weight), (node, weight)] on the flat node index."""
    di, dj = dirn
    T = i * ngy + j
    C = T + di * ngy + dj
    g = (i + 1 + di) * SY + (j + 1 + dj)
    one, two = F(1), F(2)
    if dirn == (0, 1):
        d = x - vx / vy * y
        return [(C, one - d), (C + ngy, d)]
    if dirn == (0, -1):
        d = x + vx / vy * (one - y)
        return [(T, one - d), (T + ngy, d)]
    if dirn == (1, 0):
        d = y - vy / vx * x
        return [(C, one - d), (C + 1, d)]
    if dirn == (-1, 0):
        d = y + vy / vx * (one - x)
        return [(T, one - d), (T + 1, d)]
    if dirn == (1, 1):
        d = x - vx / vy * y
        if d >= 0:
            if SI[g - 1]:
                d = y - vy / vx * x
                return [(C - 1, -d), (C, one + d)]
            return [(C, one - d), (C + ngy, d)]
        if SI[g - SY]:
            return [(T + 1, -d), (C, one + d)]
        d = y - vy / vx * x
        return [(C, one - d), (C + 1, d)]
    if dirn == (1, -1):
        d = x + vx / vy * (one - y)
        if d >= 0:
            if SI[g + 1]:
                d = y - vy / vx * x
                return [(C + 1, two - d), (C + 2, d - one)]
            return [(C + 1, one - d), (C + 1 + ngy, d)]
        if SI[g - SY]:
            return [(T, -d), (C + 1, one + d)]
        d = y - vy / vx * x
        return [(C, one - d), (C + 1, d)]
    if dirn == (-1, 1):
        d = x - vx / vy * y
        if d < 1:
            if SI[g - 1]:
                d = y + vy / vx * (one - x)
                return [(C + ngy - 1, -d), (C + ngy, one + d)]
            return [(C, one - d), (C + ngy, d)]
        if SI[g + SY]:
            return [(T + 1, two - d), (T + 1 + ngy, d - one)]
        d = y + vy / vx * (one - x)
        return [(T + 1, one - d), (T + 2, d)]
    d = x + vx / vy * (one - y)  # (-1, -1)
    if d < 1:
        if SI[g + 1]:
            d = y + vy / vx * (one - x)
            return [(T, two - d), (T + 1, d - one)]
        return [(C, one - d), (T, d)]
    if SI[g + SY]:
        return [(T, two - d), (T + ngy, d - one)]
    d = y + vy / vx * (one - x)
    return [(T - 1, one - d), (T, d)]


def setup_case():
    S = hpic.Setup(dielectric_deck(), seed=4343)
    assert S.info.n_dielectric == 2
    o = oracle.from_setup(S, 32)
    info = S.info
    for s in range(info.nsp):
        z = np.zeros(0, np.float32)
        o.set_particles(s, np.zeros(info.Csize, np.int32), z, z, z, z, z)
    return S, o


def place(S, o):
    info = S.info
    cells = np.array([i * info.ncy + j for i, j, *_ in CROSSINGS])
    order = np.argsort(cells, kind="stable")
    counts = np.bincount(cells, minlength=info.Csize).astype(np.int32)
    sc = S.table("scalars")
    dt, dx, dy = float(sc[0]), float(sc[3]), float(sc[4])
    x = np.array([c[3] for c in CROSSINGS], np.float32)[order]
    y = np.array([c[4] for c in CROSSINGS], np.float32)[order]
    vx = np.array([c[5] * dx / dt for c in CROSSINGS], np.float32)[order]
    vy = np.array([c[6] * dy / dt for c in CROSSINGS], np.float32)[order]
    vz = np.zeros(len(CROSSINGS), np.float32)
    o.set_particles(0, counts, x, y, vx, vy, vz)
    o.set_grid("EX", np.zeros(info.Gsize, np.float32))
    o.set_grid("EY", np.zeros(info.Gsize, np.float32))
    return [CROSSINGS[k] for k in order]


def test_split_matches_the_reference_rule():
    S, o = setup_case()
    info = S.info
    placed = place(S, o)
    o.Move()
    counts, (mx, my, mvx, mvy, _), codes = o.movers(0)
    assert codes.size == len(CROSSINGS) and np.all(codes == 15), "every placed particle enters a dielectric"
    SI = S.table("sidx")
    want = np.zeros(info.nsp * info.Gsize, np.int64)
    for k, (i, j, dirn, *_r) in enumerate(placed):
        for node, w in share(dirn, i, j, mx[k], my[k], mvx[k], mvy[k], SI, info.ngy, info.ncy + 2):
            w = F(w)
            if 0 <= node < info.Gsize and abs(w) < 2 ** 20:
                want[node] += int(np.rint(np.float64(w) * FRAC))
    assert np.all(o.grid("SURFACE_CHARGE") == 0), "the split belongs to SortBoundary"
    o.SortBoundary()
    got = o.grid("SURFACE_CHARGE")
    assert np.array_equal(got, want)
    # each crossing leaves one particle weight (the one whose node is off
    # the grid leaves part of it)
    total = got.sum() / FRAC
    assert abs(total - len(CROSSINGS)) < 1.0 and total > len(CROSSINGS) - 1


def test_source_carries_the_surface_charge():
    S, o = setup_case()
    info = S.info
    place(S, o)
    o.Move()
    o.SortBoundary()
    sig = o.grid("SURFACE_CHARGE").reshape(info.nsp, -1)
    o.Deposit()
    mode = S.table("sig_mode")
    area = S.table("area")
    qd = S.table("species").reshape(-1, 16)[:, 3].astype(np.float64)
    q = (sig.astype(np.float64) / FRAC * qd[:, None]).sum(0)
    src = o.grid("SOURCE")
    den = o.grid("DEN").reshape(info.nsp, -1)
    rho = (den * qd[:, None]).sum(0)
    on = (mode == 1) | (mode == 2)
    assert np.abs(q[on]).max() > 0
    np.testing.assert_allclose(src[on], (rho[on] + q[on]) / 8.8542e-12, rtol=1e-12, atol=0)
    np.testing.assert_allclose(src[~on], rho[~on] / 8.8542e-12, rtol=1e-12, atol=0)
    sigma = o.grid("SIGMA")
    np.testing.assert_allclose(sigma[on], np.where(mode[on] == 2, 2.0, 1.0) * q[on] / area[on], rtol=1e-12)
    # conductor-class nodes clear their surface weights
    after = o.grid("SURFACE_CHARGE").reshape(info.nsp, -1)
    assert np.all(after[:, mode == 3] == 0)


def test_surface_charge_builds_up_over_steps():
    """Electrons reach the slab first: after a few steps the slab's top
    surface holds net negative charge and the totals are whole weights."""
    S = hpic.Setup(dielectric_deck(), seed=4343)
    o = oracle.from_setup(S, 32)
    o.DepositBasic()
    o.run(0, 30, accumulate=False)
    info = S.info
    sig = o.grid("SURFACE_CHARGE").reshape(info.nsp, -1)
    assert sig[0].sum() > 0
    mode = S.table("sig_mode")
    qd = S.table("species").reshape(-1, 16)[:, 3].astype(np.float64)
    q = (sig.astype(np.float64) / FRAC * qd[:, None]).sum(0)
    assert q[(mode == 1) | (mode == 2)].sum() < 0


def test_deck_errors():
    import pytest
    for bad, msg in (
        ({"M_ID": 0}, "M_ID"),
        ({"M_ID": 1}, "duplicated"),
        ({"X1": 40}, "X1"),
        ({"Y0": 5, "Y1": 2}, "Y0 > Y1"),
        ({"M_ID": 120}, "1..99"),
    ):
        d = dielectric_deck()
        d["Geometry"]["DielectricSpec"][0].update(bad)
        with pytest.raises(hpic.HpicError, match=msg):
            hpic.Setup(d, seed=1)
    d = dielectric_deck()
    d["Geometry"]["DielectricSpec"][0]["M_ID"] = 5
    with pytest.raises(hpic.HpicError, match="in order"):
        hpic.Setup(d, seed=1)
