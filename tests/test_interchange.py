"""A case's state in the reference's own device structs (GCP, GPG, GGA of
inc/def.h): the record sizes equal the reference's, exported particles sit
where the reference keeps them (the pinning harness's layout converter,
oracle/refk.py, which follows src/cuda_Move.cu:195), an export and import
round trip is exact, and the GGA records carry the case's tables and
fields."""
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(REPO, "hybrid-final_b200"))
sys.path.insert(0, os.path.join(REPO, "oracle"))

import hpic  # noqa: E402
from hpic.decks import block_deck, ccp_deck  # noqa: E402

GOLD = os.path.join(REPO, "tests", "golden", "setup_ar_block_33x21.npz")


def test_records_have_the_reference_sizes():
    # GGA as the golden dumps of the reference's own set-up store it (56 bytes)
    z = np.load(GOLD)
    assert hpic.GGA_DTYPE.itemsize == 56 and "gga_Ex" in z.files
    assert hpic.GCP_DTYPE.itemsize == 24 and hpic.GPG_DTYPE.itemsize == 40


def test_arguments_are_checked():
    L = hpic.lib()
    assert L.hp_export_gcp(None, 0, 8, None, None) == hpic.HP_ERR_ARG
    assert L.hp_import_gcp(None, 0, 8, None, None) == hpic.HP_ERR_ARG
    assert L.hp_export_gga(None, None) == hpic.HP_ERR_ARG


@pytest.mark.gpu
def test_gcp_export_import_round_trip_and_layout():
    import refk
    case = hpic.Case(deck=ccp_deck(33, 17, 0.01, 0.005, ppc=12, voltage=150.0), seed=4)
    case.step(5)
    mpnc = max(case.info.cap[:case.info.nsp]) // 2
    info = case.info
    species = [case.particles(s) for s in range(info.nsp)]
    st = refk.to_ref(info, mpnc, species)  # the reference layout, built independently
    for s in range(info.nsp):
        gcp, gpg = case.export_gcp(s, mpnc)
        blk = slice(s * st.maxnp, s * st.maxnp + mpnc * info.Gsize)
        for q, f in enumerate(("x", "y", "vx", "vy", "vz")):
            assert np.array_equal(gcp[f].view(np.uint32), st.a[q][blk].view(np.uint32)), f
        assert np.array_equal(gpg["PtNumInCell"], st.pnc[s * info.Gsize:(s + 1) * info.Gsize])
        assert np.array_equal(gpg["den"], case.grid("DEN").reshape(info.nsp, -1)[s].astype(np.float32))
    # round trip into a second case of the same deck
    other = hpic.Case(deck=ccp_deck(33, 17, 0.01, 0.005, ppc=12, voltage=150.0), seed=9)
    for s in range(info.nsp):
        other.import_gcp(s, mpnc, *case.export_gcp(s, mpnc))
        (c1, a1), (c2, a2) = case.particles(s), other.particles(s)
        assert np.array_equal(c1, c2)
        for u, v in zip(a1, a2):
            assert np.array_equal(u.view(np.uint32), v.view(np.uint32))
    # too few slots per cell is refused
    with pytest.raises(hpic.HpicError) as e:
        case.export_gcp(0, 1)
    assert e.value.status == hpic.HP_ERR_CAPACITY


@pytest.mark.gpu
def test_gga_records_carry_tables_and_fields():
    case = hpic.Case(deck=block_deck(), seed=3)
    case.step(3)
    gga = case.export_gga()
    assert np.array_equal(gga["Boundary"], case.table("boundary"))
    assert np.array_equal(gga["CondID"], case.table("cond_id"))
    assert np.array_equal(gga["Face"], case.table("face"))
    assert np.array_equal(gga["Area"], case.table("area"))
    assert np.array_equal(gga["Ex"], case.grid("EX")) and np.array_equal(gga["Ey"], case.grid("EY"))
    assert np.array_equal(gga["Pois_Pot"], case.grid("PHI_POIS"))
    assert np.allclose(gga["Lap_Pot"] + gga["Pois_Pot"], case.grid("PHI"), rtol=0, atol=1e-4)
    # the golden GGA of the reference's set-up: the geometry columns agree
    z = np.load(GOLD)
    for f in ("Boundary", "CondID", "Face", "DensRegion", "Area"):
        assert np.array_equal(gga[f], z["gga_" + f]), f
