"""Generate the set-up golden fixtures from the reference's own code.

Runs oracle/_ref/ref_dump (the reference's src/start.c, src/load.c,
src/PhysicsData.c, src/Particle.c, src/Efield.c compiled in place by
`make -C oracle ref`) on small decks and stores every table it produces in
tests/golden/setup_<name>.npz together with the deck text and seed.  Needs
the reference tree, so it runs only where that exists; the .npz files are
committed and the tests read only them.

usage: python tests/golden/make_golden.py [--fluid] [deck names]
"""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "hybrid-final_b200"))
from hpic.decks import block_deck, ccp_deck, dielectric_deck  # noqa: E402

GGA = np.dtype([("Boundary", "i4"), ("CondID", "i4"), ("Face", "i4"), ("DensRegion", "i4"), ("Area", "f4"),
                ("Temp", "f4"), ("BackDen1", "f4"), ("BackVel1", "f4"), ("BackDen2", "f4"), ("BackVel2", "f4"),
                ("Lap_Pot", "f4"), ("Pois_Pot", "f4"), ("Ex", "f4"), ("Ey", "f4")])


DECKS = {
    "ar_17x9": (ccp_deck(17, 9, 0.005, 0.0025, ppc=10), 12345),
    "ar_33x17": (ccp_deck(33, 17, 0.01, 0.005, ppc=20, pressure_torr=0.1, voltage=200.0), 777),
    "ar_block_33x21": (block_deck(), 4242),
    # an R-L-C on the driven electrode and a capacitor on the floating block (src/Efield.c:70-78)
    "ar_circuit_33x21": (block_deck(circuits=[(50.0, 1e-6, 1e-9), (0.0, 0.0, 1.0), (2.0, 0.0, 1e-12)], ppc=16,
                                    voltage=200.0), 4444),
    "ar_diel_33x21": (dielectric_deck(), 4343),
    "aro2_33x17": (ccp_deck(33, 17, 0.01, 0.005, gas="ArO2", ppc=12, pressure_torr=0.1, voltage=200.0, te_ev=3.0,
                            ion_density={"Ar+": 1e15, "O2+": 2e14, "O+": 0.0, "O-": 2e14}), 515),
    "o2_33x17": (ccp_deck(33, 17, 0.01, 0.005, gas="O2", ppc=12, pressure_torr=0.1, voltage=200.0, te_ev=3.0,
                          ion_density={"O2+": 1e15, "O+": 1e14, "O-": 1e14}), 616),
    # the reference's other load types (src/Particle.c:52-175)
    "ar_33x17_exp": (ccp_deck(33, 17, 0.01, 0.005, ppc=20, load_type=1, load_pos=(0.005, 0.003, 0.002, 0.0025)), 31),
    "ar_33x17_cos": (ccp_deck(33, 17, 0.01, 0.005, ppc=20, load_type=2, load_pos=(0.005, 0.006, 0.004, 0.0025)), 32),
    "ar_33x17_npr": (ccp_deck(33, 17, 0.01, 0.005, ppc=20, load_type=3, load_pos=(0.002, 0.008, 0.001, 0.004),
                              ratio=5), 33),
}


def dump(name, deck, seed):
    exe = os.path.join(REPO, "oracle", "_ref", "ref_dump")
    if not os.path.exists(exe):
        subprocess.run(["make", "-C", os.path.join(REPO, "oracle"), "ref"], check=True)
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "deck.json")
        with open(path, "w") as f:
            json.dump(deck, f)
        out = os.path.join(tmp, "out")
        os.makedirs(out)
        subprocess.run([exe, path, str(seed), out], check=True, stdout=subprocess.DEVNULL)
        meta = dict(line.split() for line in open(os.path.join(out, "meta.txt")))
        arrs = {}
        for fn in os.listdir(out):
            if not fn.endswith(".bin"):
                continue
            key = fn[:-4]
            if key == "gga":
                g = np.fromfile(os.path.join(out, fn), dtype=GGA)
                for field in GGA.names:
                    arrs["gga_" + field] = g[field]
                continue
            dt = np.int32 if key in ("sidx", "aidx", "ai", "aj") or key.endswith("_cell") else np.float32
            arrs[key] = np.fromfile(os.path.join(out, fn), dtype=dt)
        np.savez_compressed(os.path.join(HERE, f"setup_{name}.npz"), deck=json.dumps(deck), seed=seed,
                            meta=json.dumps(meta), **arrs)


# decks whose fluid set-up and continuity solve are pinned (fluid_<name>.npz)
FLUID = ["ar_33x17", "ar_block_33x21", "o2_33x17", "aro2_33x17", "ar_33x17_exp", "ar_33x17_cos"]
FLUID_STEPS = 5


# initial fluid densities of the pinned decks (the deck builder leaves them 0)
FLUID_DENSITY = {"Ar*": 1e16, "O2A": 1e17, "O2B": 1e16, "OP": 1e18, "OD": 1e15}


def with_fluid_density(deck):
    d = json.loads(json.dumps(deck))

    def walk(o):
        if isinstance(o, dict):
            for k, v in o.items():
                if k in FLUID_DENSITY and isinstance(v, dict) and "Density" in v:
                    v["Density"] = FLUID_DENSITY[k]
                else:
                    walk(v)
        elif isinstance(o, list):
            for v in o:
                walk(v)

    walk(d)
    # the exponential and cosine decks load the fluid species the same way
    gas = d["GasSpecies"]
    if gas["ChargeSpecies"]["Loadtype"] in (1, 2):
        gas["NeutralSpecies"]["Loadtype"] = gas["ChargeSpecies"]["Loadtype"]
        gas["NeutralSpecies"]["LoadPosition(m)"] = dict(gas["ChargeSpecies"]["LoadPosition(m)"])
    return d


def dump_fluid(name, deck, seed):
    """The reference's fluid set-up (Fluid_Setting, Cal_D_*, the Gummel
    coefficients, the initial fluxes) and FLUID_STEPS steps of its
    Solve_Continuity_eqn, through ref_dump's temps/src arguments.  The gas
    temperature per node is this library's solve of the reference's own
    temperature system (the reference solves it on the GPU); the sources are
    a seeded field of the size the collision rates give."""
    import hpic
    exe = os.path.join(REPO, "oracle", "_ref", "ref_dump")
    deck = with_fluid_density(deck)
    S = hpic.Setup(deck, seed=seed, gas_temp_mode=0)
    temps = S.table("node_temp").astype(np.float32)
    nf, C = int(S.table("fluid_scalars")[3]), S.info.Csize
    rng = np.random.default_rng(seed)
    src = (rng.normal(0.0, 1.0, nf * C) * 10 ** rng.uniform(19, 22, nf * C)).astype(np.float32)
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "deck.json")
        with open(path, "w") as f:
            json.dump(deck, f)
        out = os.path.join(tmp, "out")
        os.makedirs(out)
        temps.tofile(os.path.join(tmp, "temps.bin"))
        src.tofile(os.path.join(tmp, "src.bin"))
        subprocess.run([exe, path, str(seed), out, os.path.join(tmp, "temps.bin"), os.path.join(tmp, "src.bin"),
                        str(FLUID_STEPS)], check=True, stdout=subprocess.DEVNULL)
        arrs = {}
        for fn in os.listdir(out):
            if fn.startswith("fl_"):
                dt = np.int32 if fn.endswith("lines.bin") else np.float32
                arrs[fn[:-4]] = np.fromfile(os.path.join(out, fn), dtype=dt)
    np.savez_compressed(os.path.join(HERE, f"fluid_{name}.npz"), deck=json.dumps(deck), seed=seed, temps=temps,
                        src=src, nsteps=FLUID_STEPS, **arrs)


if __name__ == "__main__":
    only = set(sys.argv[1:])  # names to (re)generate; all when none are given
    fluid_only = "--fluid" in only  # the fluid fixtures alone
    only.discard("--fluid")
    for name, (deck, seed) in DECKS.items():
        if only and name not in only:
            continue
        if not fluid_only:
            dump(name, deck, seed)
            print("wrote", name)
        if name in FLUID:
            dump_fluid(name, deck, seed)
            print("wrote fluid", name)
