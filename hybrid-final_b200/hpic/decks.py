"""Case decks in the reference's JSON case format.

Every deck written here is a valid input for the reference's own reader
(src/start.c:19-1430): same object names, same keys, same units.  The decks
describe a capacitively coupled plasma (CCP) between two plate electrodes:

* conductor M_ID 1 is node row y = 0, driven by the RF source;
* conductor M_ID 2 is node row y = NumGridy-1, grounded;
* the side walls x = 0 and x = NumGridx-1 are Neumann lines (B.C 2) over the
  rows between the electrodes (src/start.c:1491-1506 applies them).

The reader demands at least four "BoundaryCondition" lines
(src/start.c:53-56).  The two electrode rows therefore also carry a line with
B.C 3, which the geometry builder ignores (src/start.c:1495-1503 only acts on
B.C 1 and 2), so those rows stay conductor nodes.
"""
import json
import math

ARGON_CASE = [
    "0.e+Ar>e+Ar", "1.e+Ar>e+Ar*", "2.e+Ar>e+Ar*m", "3.e+Ar>2e+Ar^",
    "4.e+Ar*m>2e+Ar^", "5.Ar+Ar^>Ar^+Ar", "6.Ar+Ar^>Ar+Ar^", "7.e+Ar*m>e+Ar",
    "8.Ar*m+Ar>e+Ar^+Ar", "9.Ar+Ar*m>Ar+Ar",
]

KB_EV = 8.617333e-5  # eV per K


def _channels(names):
    return {n: 1.0 for n in names}


def _channel_keys(gas):
    """Deck keys of the O2 or Ar/O2 reaction set (the library's channel list)."""
    import os
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "data",
                        "channels_o2.txt" if gas == "O2" else "channels_aro2.txt")
    keys = []
    for line in open(path):
        if line.startswith("#") or not line.strip():
            continue
        keys.append(line.rstrip("\n").split("\t")[1])
    return keys


def ccp_deck(ngx, ngy, xlen, ylen, *, gas="Ar", pressure_torr=0.05, voltage=100.0,
             freq=13.56e6, steps_per_cycle=400, ppc=50, density=1e15, te_ev=2.0,
             ti_ev=0.026, gas_k=300.0, max_np_factor=4, aro2_ratio=(80, 20),
             ion_density=None, pcg_tol=1e-3, smoothing=0, load_type=0, load_pos=None, ratio=1,
             power_w=0.0, pd_interval=5.0, average_iter=None, circuit=None):
    """Build one CCP deck.

    ppc is the macro-particles per cell per species at `density`; np2c is
    chosen so that the reference loader's integer n_per_cell
    (src/Particle.c:10) comes out at exactly ppc.  circuit = (R, L, C)
    puts that series R-L-C between the powered electrode and its source
    (the reference's external circuit); None keeps R = L = 0, C = 1 F on
    both electrodes, which the reference reads as no circuit.
    """
    dx = xlen / (ngx - 1)
    dy = ylen / (ngy - 1)
    np2c = density * dx * dy / (ppc + 0.005)
    gsize = ngx * ngy
    max_np = int(max_np_factor * ppc * gsize)
    max_np = max(max_np, 32 * gsize)
    gas_ev = gas_k * KB_EV
    bc = [
        {"X0": 0, "X1": 0, "Y0": 1, "Y1": ngy - 2, "B.C": 2, "Temp": gas_k},
        {"X0": ngx - 1, "X1": ngx - 1, "Y0": 1, "Y1": ngy - 2, "B.C": 2, "Temp": gas_k},
        {"X0": 0, "X1": ngx - 1, "Y0": 0, "Y1": 0, "B.C": 3, "Temp": gas_k},
        {"X0": 0, "X1": ngx - 1, "Y0": ngy - 1, "Y1": ngy - 1, "B.C": 3, "Temp": gas_k},
    ]
    r_, l_, c_ = circuit if circuit is not None else (0.0, 0.0, 1.0)
    cond = [
        {"M_ID": 1, "X0": 0, "X1": ngx - 1, "Y0": 0, "Y1": 0, "Temp": gas_k,
         "R(Ohm)": float(r_), "L(H)": float(l_), "C(F)": float(c_)},
        {"M_ID": 2, "X0": 0, "X1": ngx - 1, "Y0": ngy - 1, "Y1": ngy - 1, "Temp": gas_k,
         "R(Ohm)": 0.0, "L(H)": 0.0, "C(F)": 1.0},
    ]
    src = [{"M_ID": 1, "DC(V)": 0, "Power(W)": power_w, "AC(V)": voltage, "Freq(1/s)": freq,
            "Phase(deg)": 0.0}]
    load = {"X0": 0.0, "X1": xlen, "Y0": 0.0, "Y1": ylen}
    gas_type = {"Ar": 0, "O2": 1, "ArO2": 2}[gas]
    ratio_ar, ratio_o2 = aro2_ratio if gas == "ArO2" else (100, 0)
    neutral = {"Loadtype": 0, "LoadPosition(m)": dict(load)}
    for name in ("Ar*", "O2A", "O2B", "OP", "OD"):
        neutral[name] = {"Density": 0.0, "Temp(eV)": 0.026, "Quenching": 1.0}

    def sp(sid, dens, temp):
        return {"S_ID": sid, "Density": dens, "Temp(eV)": temp, "np2c": np2c, "Ratio": ratio,
                "Max_np": max_np}

    ion = density if ion_density is None else ion_density
    # charged load (src/Particle.c:3-175): 0 uniform in the window, 1 Gaussian
    # and 2 cosine profiles (X0/Y1 centres, X1/Y0 widths), 3 Ratio per cell in
    # the window
    cload = dict(load) if load_pos is None else dict(zip(("X0", "X1", "Y0", "Y1"), load_pos))
    charge = {"Loadtype": load_type, "LoadPosition(m)": cload,
              "Electron": sp(0, density, te_ev), "Ar+": sp(1, ion.get("Ar+", density) if isinstance(ion, dict) else ion, ti_ev)}
    if gas in ("O2", "ArO2"):
        dens = ion if isinstance(ion, dict) else {}
        base = 2 if gas == "ArO2" else 1  # species order: e, (Ar+), O2+, O+, O-
        charge["O2+"] = sp(base, dens.get("O2+", 0.0), ti_ev)
        charge["O+"] = sp(base + 1, dens.get("O+", 0.0), ti_ev)
        charge["O-"] = sp(base + 2, dens.get("O-", 0.0), ti_ev)
    deck = {
        "GPU_Device_Number": {"GPUDevice": 0},
        "Geometry": {
            "SystemSpec": {"X_length(m)": xlen, "Y_length(m)": ylen, "Z_length(m)": 1.0,
                           "NumGridx": ngx, "NumGridy": ngy},
            "BoundaryCondition": bc, "ConductorSpec": cond, "Source": src, "DielectricSpec": [],
        },
        "GasSpecies": {
            "Type(0:Ar,1:O2,2:Ar/O2)": gas_type,
            "TotalPres(Torr)": pressure_torr,
            "Background": {"Argon": {"Ratio": ratio_ar, "Temp(eV)": gas_ev},
                           "Oxygen": {"Ratio": ratio_o2, "Temp(eV)": gas_ev}},
            "NeutralSpecies": neutral,
            "ChargeSpecies": charge,
        },
        "SimulationMethod": {
            "TimeStep_PIC": steps_per_cycle, "TimeStep_Conti": 200,
            "FieldTest": {"Laplace_Test_Flag": 0, "Laplace_Field_Solver": 8, "Laplace_Field_Tec_Save": 0},
            "PCGMarginOfError": pcg_tol, "HistoryMax": 1000000, "HistoryDivide": 4,
            "AverageIter": steps_per_cycle if average_iter is None else average_iter,
            "DensitySmoothing": smoothing,
            "ParticleLimit": max_np, "ConstB_Flag": 0,
            "ContinuitySteadyState": {"Flag": 0, "Check": 1, "Margin": 1.0},
            "PowerDrivenOption": {"Interval": pd_interval, "VoltageUpDownRatio": 0.05},
            "SimulationStop": {"EndTime(s)": 1e-3,
                               "SteadyStatePrint": {"Flag": 0, "AveMargin(%)": 0.05, "SatGoal": 50}},
        },
        "Diagnostics": {
            "BasicDiagnostic": 0, "MassRatio": 1.0,
            "TecplotSave": {
                "Initial_Setting": {"Init_Gsize_Save": 0, "Init_CXdata_Save": 0,
                                    "Init_Particle_Save": 0, "Init_Particle_Num": 0},
                "Tecplot2D": 0, "Tec_1Cycle_Movie_Interval": 0, "Tec_1Cycle_Movie_FrameNum": 50,
                "Tec_1Cycle_Movie_PT_Interval": 0, "Tec_1Cycle_Movie_PT_FrameNum": 50,
                "Tec_Movie": {"Flag": 0, "Term": 20, "FrameNum_per_Cycle": 8, "Interval": 10},
                "Tec_Ave_Movie": 0, "Tec_Ave_Movie_Interval": 1, "Tec_Ave_Movie_num": 100,
            },
            "DumpFileSave": {"Cycle": [{"Start": 0.0, "End": 1.0e9, "Term": 1.0e9}]},
        },
        "Collision_On_Off": {
            "ArgonCase": _channels(ARGON_CASE),
            "OxygenCase": _channels(_channel_keys("O2")) if gas == "O2" else {},
            "Argon/OxygenCase": _channels(_channel_keys("ArO2")) if gas == "ArO2" else {},
        },
    }
    return deck


def block_deck(circuits=None, ppc=8, voltage=100.0, max_np_factor=4):
    """A 33 x 21 CCP with thick block electrodes (node rows 0-2 and 18-20)
    and a floating block conductor inside (nodes 12-18 x 8-11): exercises the
    conductor-face classification and the >= 100 StructureIndex codes, so
    particles are absorbed on (and counted for) conductors.  circuits: an
    (R, L, C) per conductor (M_ID 1, 2, 3), the reference's external circuit;
    None is R = L = 0, C = 1 F everywhere (no circuit)."""
    d = ccp_deck(33, 21, 0.01, 0.00625, ppc=ppc, voltage=voltage, max_np_factor=max_np_factor)
    geo = d["Geometry"]
    rlc = circuits or [(0.0, 0.0, 1.0)] * 3
    geo["ConductorSpec"] = [
        {"M_ID": 1, "X0": 0, "X1": 32, "Y0": 0, "Y1": 2, "Temp": 300.0},
        {"M_ID": 2, "X0": 0, "X1": 32, "Y0": 18, "Y1": 20, "Temp": 300.0},
        {"M_ID": 3, "X0": 12, "X1": 18, "Y0": 8, "Y1": 11, "Temp": 350.0},
    ]
    for c, (r_, l_, c_) in zip(geo["ConductorSpec"], rlc):
        c.update({"R(Ohm)": float(r_), "L(H)": float(l_), "C(F)": float(c_)})
    geo["BoundaryCondition"] = [
        {"X0": 0, "X1": 0, "Y0": 0, "Y1": 20, "B.C": 2, "Temp": 300.0},
        {"X0": 32, "X1": 32, "Y0": 0, "Y1": 20, "B.C": 2, "Temp": 300.0},
        {"X0": 0, "X1": 32, "Y0": 0, "Y1": 0, "B.C": 1, "Temp": 300.0},
        {"X0": 0, "X1": 32, "Y0": 20, "Y1": 20, "B.C": 1, "Temp": 300.0},
    ]
    return d


def dielectric_deck(ppc=8, voltage=200.0):
    """A 33 x 21 CCP whose driven electrode (node row 0) is covered by a
    dielectric slab (M_ID 3, eps_r 4, node rows 0-3 across the whole width, so
    it meets both Neumann side walls) with a floating dielectric block inside
    (M_ID 4, eps_r 3.9, nodes 12-18 x 9-12): exercises the dielectric faces and
    areas, the 1..99 StructureIndex codes, the surface-charge split of
    SortBoundary for straight and diagonal crossings, and SumSource's interior
    and wall classes."""
    d = ccp_deck(33, 21, 0.01, 0.00625, ppc=ppc, voltage=voltage)
    d["Geometry"]["DielectricSpec"] = [
        {"M_ID": 3, "X0": 0, "X1": 32, "Y0": 0, "Y1": 3, "Epsilon": 4.0},
        {"M_ID": 4, "X0": 12, "X1": 18, "Y0": 9, "Y1": 12, "Epsilon": 3.9},
    ]
    return d


def write_deck(path, deck):
    with open(path, "w") as f:
        json.dump(deck, f, indent=1)
