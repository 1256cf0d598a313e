"""The bench's reference arm builds its case with the reference's own set-up
code (oracle/_ref/ref_dump) and oracle/refsetup.py, without this library.  On
the same deck and seed every table the oracle reads must equal the library's
set-up (itself pinned to the reference in test_setup.py): bit for bit, but
for the per-cell collision probabilities, whose 1 - exp(.) may differ by one
float ulp of the exponential between libm and NumPy."""
import numpy as np
import pytest

import hpic
import refsetup
from hpic.decks import ccp_deck

pytestmark = pytest.mark.skipif(not refsetup.available(), reason="oracle/_ref/ref_dump not built")

EXACT = ["sidx", "boundary", "face", "cond_id", "dens_region", "area", "eps_r", "xsec", "collf", "vsave", "stencil",
         "unk_node", "dep_factor", "sigv", "scalars", "sources", "lap", "back_den1", "back_vel1", "fluid_den",
         "node_temp", "a_val", "ai", "aj", "matm", "plasma_region", "fluid_cell_den", "fluid_xlines", "fluid_ylines",
         "fluid_xl_fg", "fluid_yl_fg", "fluid_D", "fluid_gax", "fluid_gbx", "fluid_gay", "fluid_gby", "fluid_flux_x0",
         "fluid_flux_y0", "fluid_scalars", "fluid_rate_f"]


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32) if a.dtype.itemsize == 4 else a


@pytest.mark.parametrize("deck,seed", [
    (ccp_deck(65, 33, 0.02, 0.01, ppc=30), 1000),
    (ccp_deck(33, 17, 0.01, 0.005, ppc=20, pressure_torr=0.5, voltage=300.0), 7),
])
def test_reference_arm_setup_equals_library_setup(deck, seed):
    R = refsetup.RefSetup(hpic.deck_text(deck), seed)
    S = hpic.Setup(deck, seed=seed, gas_temp_mode=0)
    for name in EXACT:
        assert np.array_equal(bits(R.table(name)), bits(S.table(name))), name
    # species scalars: all but the library's own slot count (column 14)
    rs, ss = R.table("species").reshape(-1, 16), S.table("species").reshape(-1, 16)
    assert np.array_equal(bits(rs[:, :14]), bits(ss[:, :14]))
    assert np.max(np.abs(R.table("prob") - S.table("prob"))) <= 1.2e-7
    for s in range(S.info.nsp):
        rc, ra = R.particles(s)
        sc, sa = S.particles(s, layout=0)
        assert np.array_equal(rc, sc)
        for a, b in zip(ra, sa):
            assert np.array_equal(bits(a), bits(b))
    for k in ("ngx", "ngy", "ncx", "ncy", "Gsize", "Csize", "nsp", "cond_numr", "n_unknowns", "mcc_stride"):
        assert getattr(R.info, k) == getattr(S.info, k), k
