"""Checkpoint and resume (hp_case_save / hp_case_load).

A case stopped after some steps, saved, and loaded into a fresh case built
from the same deck continues bit for bit as the case that was not stopped.
The file opens with the reference's V000 dump layout
(src/cuda_SaveDump.cu:5-106), checked here field by field with a reader of
that layout."""
import struct

import numpy as np
import pytest

import hpic
from hpic.decks import ccp_deck, dielectric_deck

pytestmark = pytest.mark.gpu


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32 if a.dtype.itemsize == 4 else np.uint64)


def same(a, b):
    return a.shape == b.shape and np.array_equal(bits(a), bits(b))


DECKS = {
    "ar": (ccp_deck(33, 17, 0.01, 0.005, ppc=20, pressure_torr=0.1, voltage=300.0), 777),
    "aro2": (ccp_deck(33, 17, 0.01, 0.005, gas="ArO2", ppc=20, pressure_torr=0.1, voltage=200.0, te_ev=3.0,
                      ion_density={"Ar+": 1e15, "O2+": 2e14, "O+": 0.0, "O-": 2e14}), 4242),
    "diel": (dielectric_deck(), 4343),
    "power": (ccp_deck(33, 17, 0.01, 0.005, ppc=20, power_w=0.5, pd_interval=0.02), 56),
}
CAP = {"diel": 256}
GRIDS = ("EX", "EY", "PHI", "PHI_POIS", "DEN", "SOURCE", "PCG_X", "PCG_B", "AVE_DEN", "AVE_PHI", "AVE_SOURCE",
         "AVE_EX", "AVE_EY", "MCC_COUNT", "EEDF", "SURFACE_CHARGE", "SIGMA", "SOURCE_AC", "POWER_STATE")


def read_v000_head(path, nsp):
    """t, tstep, cstep, MainGas and per species (np2c, records) of a V000 dump."""
    with open(path, "rb") as f:
        t, tstep, cstep, gas = struct.unpack("<diii", f.read(20))
        sp = []
        for _ in range(nsp):
            np2c, n = struct.unpack("<fi", f.read(8))
            rec = np.frombuffer(f.read(24 * n), dtype=[("cid", "<i4"), ("x", "<f4"), ("y", "<f4"), ("vx", "<f4"),
                                                       ("vy", "<f4"), ("vz", "<f4")])
            sp.append((np2c, rec))
    return t, tstep, cstep, gas, sp


@pytest.mark.parametrize("name", list(DECKS))
@pytest.mark.parametrize("field_mode", [0, 2])
def test_resume_is_bit_exact(tmp_path, name, field_mode):
    deck, seed = DECKS[name]
    opts = dict(field_mode=field_mode, move_mode=1, gas_temp_mode=1, eedf_every=3, cap_per_cell=CAP.get(name, 0))
    a = hpic.Case(deck, seed=seed, **opts)
    a.step(9)
    path = tmp_path / "case.dump"
    a.save(path)
    b = hpic.Case(deck, seed=seed + 1, **opts)  # the dump's seed replaces the case's
    b.load(path)
    assert b.tstep() == a.tstep() == 9
    assert b.average_count() == a.average_count()
    a.step(7)
    b.step(7)
    for s in range(a.info.nsp):
        ca, pa = a.particles(s)
        cb, pb = b.particles(s)
        assert np.array_equal(ca, cb)
        for x, y in zip(pa, pb):
            assert same(x, y)
    for g in GRIDS:
        assert same(a.grid(g), b.grid(g)), g
    assert a.pushes() == b.pushes()
    assert a.status() == b.status() == 0
    if name == "diel":
        assert a.grid("SURFACE_CHARGE").sum() > 0


def test_v000_part_holds_the_reference_records(tmp_path):
    deck, seed = DECKS["ar"]
    c = hpic.Case(deck, seed=seed, field_mode=2, move_mode=1)
    c.step(5)
    path = tmp_path / "v000.dump"
    c.save(path)
    t, tstep, cstep, gas, sp = read_v000_head(path, c.info.nsp)
    assert tstep == 5 and cstep == 0 and gas == c.info.main_gas
    assert t == pytest.approx(5 * c.info.dt, rel=1e-6)
    ngy, ncy = c.info.ngy, c.info.ncy
    for s, (np2c, rec) in enumerate(sp):
        counts, (x, y, vx, vy, vz) = c.particles(s)
        assert rec.size == counts.sum()
        cell = np.repeat(np.arange(counts.size), counts)
        i, j = cell // ncy, cell % ncy
        assert np.array_equal(rec["cid"], i * ngy + j)  # the node of the cell's lower-left corner
        assert same(rec["x"], (i.astype(np.float32) + x).astype(np.float32))
        assert same(rec["y"], (j.astype(np.float32) + y).astype(np.float32))
        assert same(rec["vz"], vz)


def test_load_refuses_another_grid(tmp_path):
    deck, seed = DECKS["ar"]
    c = hpic.Case(deck, seed=seed)
    c.step(2)
    path = tmp_path / "a.dump"
    c.save(path)
    other = hpic.Case(ccp_deck(17, 9, 0.005, 0.0025, ppc=10), seed=1)
    t0 = other.tstep()
    with pytest.raises(hpic.HpicError):
        other.load(path)
    assert other.tstep() == t0  # nothing was changed


def test_v000_sigma_is_the_dielectric_surface_charge(tmp_path):
    """The V000 per-(species, node) records (den, ave_den, sigma) carry the
    dielectric surface charge as the reference's float GPG.sigma."""
    deck, seed = DECKS["diel"]
    c = hpic.Case(deck, seed=seed, field_mode=1, move_mode=1, cap_per_cell=CAP["diel"])
    c.step(12)
    path = tmp_path / "diel.dump"
    c.save(path)
    info = c.info
    t, tstep, cstep, gas, sp = read_v000_head(path, info.nsp)
    off = 20 + sum(8 + 24 * rec.size for _, rec in sp)
    ncx, ncy, ngx, ngy, G = info.ncx, info.ncy, info.ngx, info.ngy, info.Gsize
    nfsp = 1  # the Ar set carries one fluid species (Ar*)
    off += 4 + nfsp * 4 * (2 * ncx * ncy + ngx * ncy + ncx * ngy)  # Conti_Flag, fluid arrays
    off += 3 * 4  # history counters
    raw = np.fromfile(path, dtype="<f4", count=3 * info.nsp * G, offset=off).reshape(info.nsp * G, 3)
    want = (c.grid("SURFACE_CHARGE").astype(np.float64) / 2.0 ** hpic.SIGMA_FRAC_BITS).astype(np.float32)
    assert want.sum() > 0
    assert same(raw[:, 2].copy(), want)
    assert same(raw[:, 0].copy(), c.grid("DEN").astype(np.float32))
