"""Power-driven sources (Source "Power(W)" != 0): the set-up of the
reference's Source_setting (src/Efield.c:29-66) and PowerDrivenOption
(src/start.c:786-790), and the controller of its Diagnostic
(src/cuda_Diagnostic.cu:365-420) on the oracle.  The kernels are checked
against the oracle bit for bit in test_gpu_ops (test_power_controller_bit_exact)."""
import numpy as np
import pytest

import hpic
import oracle
from hpic.decks import ccp_deck


def deck(**kw):
    return ccp_deck(33, 17, 0.01, 0.005, ppc=20, **kw)


def test_settings():
    S = hpic.Setup(deck(power_w=0.5, pd_interval=0.05), seed=5)
    assert S.info.power_driven == 1
    pw = S.table("power")
    # Interval in RF periods x 400 steps; one source, its conductor's first power source
    assert int(pw[0]) == 20 and np.isclose(pw[1], 0.05) and pw[2] == np.float32(0.5)
    assert list(pw[3:5]) == [1, 0] and list(pw[5:7]) == [0, -1]
    d = deck(power_w=0.5)
    d["SimulationMethod"]["PowerDrivenOption"] = {}
    S = hpic.Setup(d, seed=5)
    assert int(S.table("power")[0]) == 5 * 400  # the reference's default: 5 periods
    assert hpic.Setup(deck(), seed=5).info.power_driven == 0


def test_at_most_two_power_sources_per_conductor():
    d = deck(power_w=1.0)
    s0 = d["Geometry"]["Source"][0]
    d["Geometry"]["Source"] = [dict(s0), dict(s0, **{"Freq(1/s)": 2e6}), dict(s0, **{"Freq(1/s)": 1e6})]
    with pytest.raises(hpic.HpicError, match="two power-driven"):
        hpic.Setup(d, seed=5)


def test_controller_arms_then_revises():
    S = hpic.Setup(deck(power_w=0.5, pd_interval=0.05), seed=5, field_mode=2, move_mode=1)
    o = oracle.from_setup(S, 32, field_mode=2)
    o.c.move_mode = 1
    o.DepositBasic()
    amps = []
    for k in range(4):
        o.run(20 * k, 20, accumulate=False)
        amps.append(float(o.grid("SOURCE_AC")[0]))
    assert amps[0] == 100.0  # the first revision only arms the controller
    assert amps[1] != 100.0 and np.all(np.isfinite(amps))
