"""Density smoothing (DensitySmoothing > 0): the oracle's Deposit applies the
reference's 1-2-1 filter (Smooth_121_x then Smooth_121_y,
src/cuda_Deposit.cu:105-170) that many times; checked here against a direct
numpy restatement of those two kernels.  The GPU kernels are checked against
the oracle bit for bit in test_gpu_ops (deck ar_33x17_smooth2)."""
import numpy as np

import hpic
import oracle
from hpic.decks import ccp_deck


def smooth_121(v, dr, ngx, ngy, along_y):
    out = np.zeros_like(v)
    for n in range(v.size):
        x, y = divmod(n, ngy)
        at, last, step = (y, ngy - 1, 1) if along_y else (x, ngx - 1, ngy)
        a1, a2, a3 = 0, 1, 0
        if dr[n]:
            if at == 0:
                a3 = 2
            elif at == last:
                a1 = 2
            elif dr[n - step] == 0 and dr[n + step] != 0:
                a3 = 2
            elif dr[n - step] != 0 and dr[n + step] == 0:
                a1 = 2
            elif dr[n - step] == 0 and dr[n + step] == 0:
                a2 = 4
            else:
                a1 = a3 = 1
        else:
            a2 = 0
        left = a1 * v[n - step] if a1 else 0.0
        right = a3 * v[n + step] if a3 else 0.0
        out[n] = 0.25 * (left + (2 * a2) * v[n] + right)
    return out


def test_oracle_deposit_smooths_as_the_reference():
    S = hpic.Setup(ccp_deck(33, 17, 0.01, 0.005, ppc=20, smoothing=2), seed=778)
    assert S.info.n_smt == 2
    o = oracle.from_setup(S, 32)
    o.DepositBasic()
    raw = o.grid("DEN").reshape(S.info.nsp, -1).copy()
    o.Deposit()
    got = o.grid("DEN").reshape(S.info.nsp, -1)
    dr = S.table("dens_region", np.int32)
    for s in range(S.info.nsp):
        v = raw[s]
        for _ in range(2):
            v = smooth_121(smooth_121(v, dr, S.info.ngx, S.info.ngy, False), dr, S.info.ngx, S.info.ngy, True)
        assert np.array_equal(v.view(np.uint64), got[s].view(np.uint64))
    assert not np.array_equal(raw, got)
    assert np.all(np.isfinite(o.grid("SOURCE")))
