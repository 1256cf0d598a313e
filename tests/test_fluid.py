"""The fluid (metastable and radical) species against the reference's own code.

tests/golden/fluid_<deck>.npz holds, for six decks (Ar, Ar with a blocking
electrode, O2, Ar/O2, and the exponential and cosine loads), the reference's
host-side fluid set-up (Fluid_Setting, Set_Con_Region, Set_Con_Boundary, the
diffusion coefficients, the Gummel coefficients, the initial fluxes) and its
state after 5 calls of Solve_Continuity_eqn on a seeded source field, written
by the reference's src/Fluid.c and src/cuda_Fluid.cu compiled unedited
(tests/golden/make_golden.py, oracle/ref_fluid.cu).  The library's set-up
tables and the oracle's continuity solve must equal them bit for bit."""
import json

import numpy as np
import pytest

import hpic
import oracle

DECKS = ["ar_33x17", "ar_block_33x21", "o2_33x17", "aro2_33x17", "ar_33x17_exp", "ar_33x17_cos"]
TABLES = dict(fl_xlines="fluid_xlines", fl_ylines="fluid_ylines", fl_xl_fg="fluid_xl_fg", fl_yl_fg="fluid_yl_fg",
              fl_D="fluid_D", fl_den0="fluid_cell_den", fl_gax="fluid_gax", fl_gbx="fluid_gbx", fl_gay="fluid_gay",
              fl_gby="fluid_gby", fl_flux_x0="fluid_flux_x0", fl_flux_y0="fluid_flux_y0")


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32) if a.dtype == np.float32 else a


def load(name):
    z = np.load(f"{__file__.rsplit('/', 1)[0]}/golden/fluid_{name}.npz")
    deck = json.loads(str(z["deck"]))
    S = hpic.Setup(deck, seed=int(z["seed"]), gas_temp_mode=0)
    # the gas temperature the golden was made with
    assert np.array_equal(bits(S.table("node_temp").astype(np.float32)), bits(z["temps"]))
    return z, S


@pytest.mark.parametrize("name", DECKS)
def test_fluid_setup_is_the_reference(name):
    z, S = load(name)
    for ref, ours in TABLES.items():
        a, b = np.asarray(S.table(ours)), z[ref]
        assert a.shape == b.shape and np.array_equal(bits(a), bits(b)), ours
    # node densities: the reference's Sync_Fluid_GFCtoGFG_forDen writes every
    # node but (0, ncy) and (ncx, 0), whose memory it never sets
    info = S.info
    node = np.asarray(S.table("fluid_den")).reshape(-1, info.ngx, info.ngy)
    ref = z["fl_node_den0"].reshape(-1, info.ngx, info.ngy)
    mask = np.ones(node.shape[1:], bool)
    mask[0, info.ncy] = mask[info.ncx, 0] = False
    assert np.array_equal(bits(node[:, mask]), bits(ref[:, mask]))
    assert not node[:, ~mask].any()


@pytest.mark.parametrize("name", DECKS)
def test_continuity_solve_is_the_reference(name):
    z, S = load(name)
    opts = hpic.CaseOpts()
    opts.seed = int(z["seed"])
    o = oracle.Oracle(S.table, S.info, opts, 32)
    o.set_grid("FLUID_SOURCE", z["src"])
    o.fluid_sweeps(int(z["nsteps"]))
    for grid, ref in (("FLUID_CELL_DEN", "fl_den"), ("FLUID_FLUX_X", "fl_flux_x"), ("FLUID_FLUX_Y", "fl_flux_y")):
        assert np.array_equal(bits(o.grid(grid)), bits(z[ref])), grid


def test_lines_cover_the_plasma_cells():
    """Every plasma cell lies on exactly one x line and one y line; a blocking
    electrode splits rows and columns into several lines."""
    z, S = load("ar_block_33x21")
    info = S.info
    plasma = np.asarray(S.table("plasma_region")).reshape(info.ncx, info.ncy) == 1
    for lines, axis in ((S.table("fluid_xlines").reshape(-1, 3), 0), (S.table("fluid_ylines").reshape(-1, 3), 1)):
        cover = np.zeros_like(plasma, int)
        for a, b, c in lines:
            if axis == 0:
                cover[a:b + 1, c] += 1
            else:
                cover[a, b:c + 1] += 1
        assert np.array_equal(cover, plasma.astype(int))
    assert len(S.table("fluid_xlines")) // 3 > plasma.any(axis=0).sum()
    assert len(S.table("fluid_ylines")) // 3 > plasma.any(axis=1).sum()
