"""Case builder vs. the reference's own set-up code (golden fixtures made by
tests/golden/make_golden.py from oracle/_ref/ref_dump).  Everything the step
consumes must match bit for bit: node classification, faces, areas,
StructureIndex, the CSR matrix and its conductor right-hand sides,
cross-section tables, the Maxwellian speed table and the seeded load."""
import glob
import json
import os

import numpy as np
import pytest

import hpic

GOLD = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "setup_*.npz")))


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32 if a.dtype.itemsize == 4 else np.uint8)


@pytest.fixture(params=GOLD, ids=[os.path.basename(p)[6:-4] for p in GOLD], scope="module")
def pair(request):
    g = np.load(request.param)
    s = hpic.Setup(str(g["deck"]), seed=int(g["seed"]))
    return s, g


def test_geometry_tables(pair):
    s, g = pair
    assert np.array_equal(s.table("sidx"), g["sidx"])
    assert np.array_equal(s.table("a_idx"), g["aidx"])
    assert np.array_equal(s.table("boundary"), g["gga_Boundary"])
    assert np.array_equal(s.table("cond_id"), g["gga_CondID"])
    assert np.array_equal(s.table("face"), g["gga_Face"])
    assert np.array_equal(s.table("dens_region"), g["gga_DensRegion"])
    assert np.array_equal(bits(s.table("area")), bits(g["gga_Area"]))


def test_cell_permittivity(pair):
    s, g = pair
    gca = np.frombuffer(g["gca"].tobytes(), dtype=np.dtype([("PlasmaRegion", "i4"), ("eps_r", "f4"), ("eps", "f4")]))
    assert np.array_equal(bits(s.table("eps_r")), bits(np.ascontiguousarray(gca["eps_r"])))


def test_surface_charge_node_classes(pair):
    """SumSource (src/cuda_Deposit.cu:35-104) reads the inward neighbour's
    class on the domain edges (x edges first) and the node's own inside."""
    s, g = pair
    b = g["gga_Boundary"].reshape(s.info.ngx, s.info.ngy)
    ngx, ngy = b.shape
    want = np.zeros_like(b)
    if len(json.loads(str(g["deck"]))["Geometry"]["DielectricSpec"]):
        for x in range(ngx):
            for y in range(ngy):
                nx, ny, edge = x, y, 1
                if x == 0: nx = 1
                elif x == ngx - 1: nx = ngx - 2
                elif y == 0: ny = 1
                elif y == ngy - 1: ny = ngy - 2
                else: edge = 0
                want[x, y] = {4: 2 if edge else 1, 3: 3}.get(int(b[nx, ny]), 0)
    assert np.array_equal(s.table("sig_mode").reshape(ngx, ngy), want)


def test_matrix(pair):
    s, g = pair
    for mine, ref in (("a_val", "a_val"), ("ta_val", "ta_val"), ("matm", "matm"), ("temp_b", "temp_b"),
                      ("cond_b", "cond_b")):
        assert np.array_equal(bits(s.table(mine)), bits(g[ref])), mine
    assert np.array_equal(s.table("ai"), g["ai"])
    assert np.array_equal(s.table("aj"), g["aj"])


def test_collision_tables(pair):
    s, g = pair
    assert np.array_equal(bits(s.table("xsec")), bits(g["xsec"]))
    assert np.array_equal(bits(s.table("collf")), bits(g["collf"]))
    assert np.array_equal(bits(s.table("vsave")), bits(g["vsave"]))


def test_scalars(pair):
    s, g = pair
    meta = json.loads(str(g["meta"]))
    sc = s.table("scalars")
    assert np.float32(sc[0]) == np.float32(float(meta["dt"]))
    spc = s.table("species").reshape(-1, 16)
    names = ["np2c", "mass", "q", "q_density", "vti", "qm", "Escale", "Ascale", "Denscale", "MCCscale"]
    for isp in range(s.info.nsp):
        for k, n in enumerate(names):
            assert np.float32(spc[isp, k]) == np.float32(float(meta[f"sp{isp}_{n}"])), (isp, n)


def test_particle_load(pair):
    s, g = pair
    for isp in range(s.info.nsp):
        cells, arrs = s.particles(isp, layout=1)
        assert np.array_equal(cells, g[f"p{isp}_cell"])
        for nm, a in zip(("x", "y", "vx", "vy", "vz"), arrs):
            assert np.array_equal(bits(a), bits(g[f"p{isp}_{nm}"])), (isp, nm)


def test_cell_sorted_load_is_the_same_particles(pair):
    s, g = pair
    for isp in range(s.info.nsp):
        counts, (x, y, vx, vy, vz) = s.particles(isp, layout=0)
        hc, (hx, hy, hvx, hvy, hvz) = s.particles(isp, layout=1)
        ix, iy = hx.astype(np.int32), hy.astype(np.int32)
        cell = ix * s.info.ncy + iy
        order = np.argsort(cell, kind="stable")
        assert np.array_equal(np.bincount(cell, minlength=s.info.Csize), counts)
        assert np.array_equal(bits(x), bits((hx - ix.astype(np.float32))[order]))
        assert np.array_equal(bits(vz), bits(hvz[order]))


def test_symmetrised_operator_is_symmetric(pair):
    """Field mode 1 solves D^-1 A x = D^-1 b with D the reference's Neumann
    doubling; the scaled operator must be symmetric."""
    s, _ = pair
    st = s.table("stencil").reshape(-1, 5)
    unk = s.table("unk_node")
    ngy, ncx, ncy = s.info.ngy, s.info.ncx, s.info.ncy
    pos = {int(n): u for u, n in enumerate(unk)}
    ii, jj = unk // ngy, unk % ngy
    d = np.where((ii == 0) | (ii == ncx), 2, 1) * np.where((jj == 0) | (jj == ncy), 2, 1)
    offs = [-ngy, -1, 0, 1, ngy]
    for u, n in enumerate(unk):
        for k, off in enumerate(offs):
            if k == 2 or st[u, k] == 0:
                continue
            v = pos[int(n) + off]
            back = 4 - k
            assert np.isclose(st[u, k] / d[u], st[v, back] / d[v], rtol=1e-6)


def test_stencil_is_the_reference_matrix(pair):
    """The field solvers apply the 5-point node stencil; every row must be the
    reference's own CSR row (src/load.c:121-246, golden a_val/ai/aj) of that
    unknown, coefficient for coefficient."""
    s, g = pair
    st = s.table("stencil").reshape(-1, 5)
    unk = s.table("unk_node")
    aidx = g["aidx"]
    ai, aj, av = g["ai"], g["aj"], g["a_val"]
    ngy = s.info.ngy
    offs = [-ngy, -1, 0, 1, ngy]
    assert unk.size == int(aidx.max())
    for u, n in enumerate(unk):
        row = int(aidx[n]) - 1
        want = {int(aj[k]) - 1: av[k] for k in range(ai[row] - 1, ai[row + 1] - 1)}
        got = {}
        for k, off in enumerate(offs):
            if k == 2 or st[u, k] != 0:
                col = int(aidx[int(n) + off]) - 1
                assert col >= 0, "stencil reaches a node that is not an unknown"
                got[col] = st[u, k]
        assert got.keys() == want.keys(), f"row {row}: columns {sorted(got)} vs {sorted(want)}"
        for col in want:
            assert bits(np.float32(got[col])) == bits(np.float32(want[col])), f"row {row} col {col}"


def test_deck_errors():
    deck = json.loads(str(np.load(GOLD[0])["deck"]))
    bad = json.loads(json.dumps(deck))
    bad["Geometry"]["BoundaryCondition"] = bad["Geometry"]["BoundaryCondition"][:3]
    with pytest.raises(hpic.HpicError) as e:
        hpic.Setup(bad)
    assert e.value.status == hpic.HP_ERR_DECK
    bad = json.loads(json.dumps(deck))
    bad["Geometry"]["ConductorSpec"][0]["M_ID"] = 2
    with pytest.raises(hpic.HpicError) as e:
        hpic.Setup(bad)
    assert e.value.status == hpic.HP_ERR_DECK
    # an R/L/C on a conductor is the external circuit (tests/test_circuit.py)
    ok = json.loads(json.dumps(deck))
    ok["Geometry"]["ConductorSpec"][0]["R(Ohm)"] = 50.0
    assert hpic.Setup(ok).info.circuit == 1
    bad = json.loads(json.dumps(deck))
    bad["SimulationMethod"]["PCGMarginOfError"] = 0
    with pytest.raises(hpic.HpicError) as e:
        hpic.Setup(bad)
    assert e.value.status == hpic.HP_ERR_DECK
    with pytest.raises(hpic.HpicError) as e:
        hpic.Setup("{ not json")
    assert e.value.status == hpic.HP_ERR_DECK
    # SMARTLOAD passes the reader, but the reference's loader exits on it
    bad = json.loads(json.dumps(deck))
    bad["GasSpecies"]["ChargeSpecies"]["Loadtype"] = 4
    with pytest.raises(hpic.HpicError) as e:
        hpic.Setup(bad)
    assert e.value.status == hpic.HP_ERR_UNSUPPORTED


def test_no_gpu_is_a_loud_error():
    from conftest import have_gpu
    if have_gpu():
        pytest.skip("a GPU is present")
    deck = str(np.load(GOLD[0])["deck"])
    with pytest.raises(hpic.HpicError) as e:
        hpic.Case(deck)
    assert e.value.status == hpic.HP_ERR_NO_CUDA


def test_gas_temperature_modes():
    """Mode 0 keeps the reference's temperature operator, which has no
    Neumann doubling on the x = 0 edge and cools the gas toward that wall;
    mode 1 solves on the potential operator and keeps equal walls uniform."""
    from hpic.decks import ccp_deck
    deck = ccp_deck(33, 17, 0.01, 0.005, ppc=2, gas_k=300.0)
    ref = hpic.Setup(deck, seed=1, gas_temp_mode=0).table("node_temp").reshape(33, 17)
    fix = hpic.Setup(deck, seed=1, gas_temp_mode=1).table("node_temp").reshape(33, 17)
    assert np.allclose(fix, 300.0, rtol=1e-5)
    assert ref[0, 8] < 0.5 * ref[16, 8]       # cold x = 0 wall
    assert abs(ref[-1, 8] - 300.0) < 10.0      # the x = ncx wall keeps its Neumann doubling
