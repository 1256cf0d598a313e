"""Seeded synthetic case mixes for the batched and served forms.

Both draw Ar CCP decks (hpic.decks.ccp_deck: plate electrodes, Neumann side
walls, 13.56 MHz, 400 steps per RF period) whose parameters vary from case to
case, so that a batch holds uneven grids and particle counts:

* batched_cases: grids uniform over {65x33, 129x65, 257x129} (2x1, 4x2, 8x4
  cm), pressure log-uniform in 10-200 mTorr, RF voltage uniform in 50-300 V,
  20-200 macro-particles per cell per species, per-case seeds;
* served_stream: Poisson arrivals, Ar or 80/20 Ar/O2 (even odds), grids over
  {65x33, 129x65, 257x129, 513x257}, the same pressure and voltage ranges,
  50-200 particles per cell, 1-10 RF periods per request.
"""
import numpy as np

from .decks import ccp_deck

GRIDS = {  # nodes -> domain size (m): the cell stays 312.5 um
    (65, 33): (0.02, 0.01),
    (129, 65): (0.04, 0.02),
    (257, 129): (0.08, 0.04),
    (513, 257): (0.16, 0.08),
}


def _case(rng, grids, ppc_range, gas="Ar", max_np_factor=8):
    g = grids[rng.integers(len(grids))]
    xlen, ylen = GRIDS[g]
    p_torr = float(np.exp(rng.uniform(np.log(0.010), np.log(0.200))))
    volts = float(rng.uniform(50.0, 300.0))
    ppc = int(rng.integers(ppc_range[0], ppc_range[1] + 1))
    extra = {}
    if gas == "ArO2":  # 80/20 Ar/O2 with the precision-form ion mix
        extra = dict(gas="ArO2", aro2_ratio=(80, 20), te_ev=3.0,
                     ion_density={"Ar+": 1e15, "O2+": 2e14, "O+": 0.0, "O-": 2e14})
    # 8x the initial count per cell: small, strongly driven cases compress the
    # plasma well beyond the load density in their first steps (16x for the
    # served stream, whose requests run up to 10 RF periods)
    deck = ccp_deck(g[0], g[1], xlen, ylen, ppc=ppc, voltage=volts, pressure_torr=p_torr,
                    max_np_factor=max_np_factor, **extra)
    desc = dict(nodes=f"{g[0]}x{g[1]}", gas=gas, pressure_torr=round(p_torr, 5), voltage=round(volts, 2), ppc=ppc)
    return deck, desc


def batched_cases(n=64, seed=2024):
    """n (deck, seed, description) triples of the batched form."""
    rng = np.random.default_rng(seed)
    grids = [(65, 33), (129, 65), (257, 129)]
    out = []
    for k in range(n):
        deck, desc = _case(rng, grids, (20, 200))
        out.append((deck, int(rng.integers(1, 2 ** 31 - 2)), desc))
    return out


def served_stream(n=512, rate_per_s=4.0, seed=7, steps_per_cycle=400, cycles=(1, 10)):
    """n requests (arrival time s, deck, nsteps, seed, description), arrivals
    a Poisson process of the given mean rate."""
    rng = np.random.default_rng(seed)
    grids = list(GRIDS)
    t = 0.0
    out = []
    for k in range(n):
        t += float(rng.exponential(1.0 / rate_per_s))
        gas = "ArO2" if rng.random() < 0.5 else "Ar"
        deck, desc = _case(rng, grids, (50, 200), gas=gas, max_np_factor=16)
        ncyc = int(rng.integers(cycles[0], cycles[1] + 1))
        desc["rf_periods"] = ncyc
        out.append((t, deck, ncyc * steps_per_cycle, int(rng.integers(1, 2 ** 31 - 2)), desc))
    return out
