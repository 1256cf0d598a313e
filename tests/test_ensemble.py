"""Precision form against FP64: time averages over a whole RF period.

The step runs with FP32 particles (cell index + FP32 offset), an FP64 charge
grid and an FP64-refined field solve.  The oracle's FP64 form runs the same
case with the same random draws entirely in double precision.  Single
trajectories decorrelate (the discharge is chaotic), so the comparison is on
the time-averaged ion density and potential over one RF period (400 steps),
as relative L2 errors; the stated tolerance is 1 %.  The electron energy
distribution (EEDF, sampled every 4th step over the period) is compared as
normalised histograms: total-variation distance at most 2 % and mean energy
within 1 %.  Every input is seeded, so the numbers below are fixed, not a
random pass/fail."""
import numpy as np
import pytest

import hpic
import oracle
from hpic.decks import ccp_deck

TOL = 0.01
EEDF_TV_TOL = 0.02
OPTS = dict(field_mode=2, gas_temp_mode=1, move_mode=1, eedf_every=4)


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def eedf_errors(h, h64):
    """(total-variation distance, relative mean-energy error) of two
    electron energy histograms; bin centres (k + 1/2) 0.25 eV."""
    p = np.asarray(h, np.float64) / float(np.sum(h))
    q = np.asarray(h64, np.float64) / float(np.sum(h64))
    e = (np.arange(p.size) + 0.5) * hpic.EEDF_DE
    return 0.5 * float(np.abs(p - q).sum()), abs(float(p @ e) / float(q @ e) - 1.0)


def fp64_averages(S, nsteps):
    o = oracle.from_setup(S, 64, field_mode=2)
    o.c.move_mode = 1
    o.DepositBasic()
    o.run(0, nsteps, accumulate=True)
    d, p, n = o.averages()
    return d.reshape(S.info.nsp, -1) / n, p / n, o.eedf()


def test_fp32_oracle_within_tolerance_of_fp64():
    """CPU: the FP32 restatement (bit-identical to the GPU kernels) against FP64."""
    S = hpic.Setup(ccp_deck(33, 17, 0.01, 0.005, ppc=60), seed=5, **OPTS)
    o = oracle.from_setup(S, 32, field_mode=2)
    o.c.move_mode = 1
    o.DepositBasic()
    o.run(0, 400, accumulate=True)
    d, p, n = o.averages()
    d32, p32 = d.reshape(S.info.nsp, -1) / n, p / n
    d64, p64, h64 = fp64_averages(S, 400)
    assert rel_l2(d32[1], d64[1]) <= TOL
    assert rel_l2(p32, p64) <= TOL
    tv, de = eedf_errors(o.eedf(), h64)
    assert tv <= EEDF_TV_TOL and de <= TOL


@pytest.mark.gpu
def test_gpu_within_tolerance_of_fp64():
    """GPU precision form (65x33 nodes, 30 particles per cell and species,
    one RF period) against the FP64 oracle."""
    deck = ccp_deck(65, 33, 0.02, 0.01, ppc=30)
    S = hpic.Setup(deck, seed=5, **OPTS)
    c = hpic.Case(setup=S, seed=5, **OPTS)
    c.step(400)
    n = c.average_count()
    d32 = c.grid("AVE_DEN").reshape(c.info.nsp, -1) / n
    p32 = c.grid("AVE_PHI") / n
    assert c.status() == 0
    d64, p64, h64 = fp64_averages(S, 400)
    err_ni, err_phi = rel_l2(d32[1], d64[1]), rel_l2(p32, p64)
    tv, de = eedf_errors(c.grid("EEDF"), h64)
    print(f"time-averaged n_i rel L2 {err_ni:.3e}, phi {err_phi:.3e}; EEDF TV {tv:.3e}, mean energy {de:.3e}")
    assert err_ni <= TOL and err_phi <= TOL
    assert tv <= EEDF_TV_TOL and de <= TOL
