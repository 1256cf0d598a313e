"""The external circuit (R-L-C on a conductor; the reference's Efield_cuda,
src/cuda_Field.cu:43-103, with Source_setting's coefficients, src/Efield.c:
70-78, and the Laplace bases' conductor charges, src/cuda_Field.cu:207-216).

CPU: the coefficients against the reference's own set-up code (golden), the
cofactor inverse of include/hp_circuit.h against the reference's compiled
cofactor(), the Laplace-basis conductor charges against a numpy statement of
Cond_Sigma_Lap, one circuit step against a line-by-line transcription of
Efield_cuda's loops (mode 0) and of the charge balance (mode 1), and the
deck rules.  GPU: the circuit decks bit-exact against the oracle, alone, in a
batch and across a checkpoint."""
import ctypes as C
import json
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(REPO, "hybrid-final_b200"))
sys.path.insert(0, os.path.join(REPO, "oracle"))

import hpic  # noqa: E402
import oracle  # noqa: E402
from hpic.decks import block_deck, ccp_deck  # noqa: E402

GOLD = os.path.join(REPO, "tests", "golden", "setup_ar_circuit_33x21.npz")
REF_KERNELS = os.path.join(REPO, "oracle", "_ref", "libref_kernels.so")
MAXC = hpic.CIRCUIT_MAX
# the golden deck's circuits: an R-L-C on the driven electrode, a resistor and
# a small capacitor on the floating block
CIRCUITS = [(50.0, 1e-6, 1e-9), (0.0, 0.0, 1.0), (2.0, 0.0, 1e-12)]
# the runs': the floating block on a capacitor alone (a resistor whose R C is
# below the time step couples to the explicit particle push unstably in
# mode 1, as it would in any explicit PIC-circuit scheme)
RUN_CIRCUITS = [(50.0, 1e-6, 1e-9), (0.0, 0.0, 1.0), (0.0, 0.0, 1e-12)]


def circuit_deck(ppc=16, voltage=200.0, circuits=RUN_CIRCUITS):
    # slots for 16x the load per cell: the driven electrode swings to a few
    # hundred volts in mode 1 and packs the sheath cells
    return block_deck(circuits=circuits, ppc=ppc, voltage=voltage, max_np_factor=16)


def test_coefficients_equal_the_reference_setup():
    z = np.load(GOLD)
    s = hpic.Setup(json.loads(str(z["deck"])), seed=int(z["seed"]))
    assert s.info.circuit == 1
    nc = s.info.cond_numr
    cc = s.table("circuit")[: 5 * nc]
    assert np.array_equal(cc.view(np.uint32), z["cc_a"].view(np.uint32))


def test_no_circuit_when_r_l_are_zero_and_c_is_large():
    s = hpic.Setup(block_deck(), seed=3)
    assert s.info.circuit == 0 and s.table("circuit").size == 0
    # the reference's rule: L < 1e-30, R < 1e-30 and C >= 1 on every line (src/start.c:173-177)
    s = hpic.Setup(block_deck(circuits=[(0.0, 0.0, 1.0), (0.0, 0.0, 0.5), (0.0, 0.0, 1.0)]), seed=3)
    assert s.info.circuit == 1


def test_more_conductors_than_the_circuit_holds_are_refused():
    d = circuit_deck(circuits=CIRCUITS)
    geo = d["Geometry"]
    for k in range(4, 6):
        geo["ConductorSpec"].append({"M_ID": k, "X0": 2 + 3 * (k - 4), "X1": 3 + 3 * (k - 4), "Y0": 6, "Y1": 7,
                                     "Temp": 300.0, "R(Ohm)": 0.0, "L(H)": 0.0, "C(F)": 1.0})
    with pytest.raises(hpic.HpicError) as e:
        hpic.Setup(d, seed=3)
    assert e.value.status == hpic.HP_ERR_UNSUPPORTED


def _ref_cofactor():
    if not os.path.exists(REF_KERNELS):
        pytest.skip("the reference's step code is not built here (make -C oracle ref_kernels)")
    L = C.CDLL(REF_KERNELS)
    f = L._Z8cofactorPPff  # cofactor(float **, float), src/cuda_Field.cu:906-941
    f.restype = None
    f.argtypes = [C.POINTER(C.POINTER(C.c_float)), C.c_float]
    return f


def test_inverse_is_the_reference_cofactor_bit_for_bit():
    cof = _ref_cofactor()
    L = oracle.lib()
    L.or_circuit_inverse.argtypes = [C.POINTER(C.c_float), C.c_int]
    rng = np.random.default_rng(11)
    for n in (2, 3, 4):
        for trial in range(300):
            m = (rng.normal(0.0, 1.0, (n, n)) * 10.0 ** rng.uniform(-12, 2)).astype(np.float32)
            if trial % 3 == 0:  # capacitance-like: diagonally dominant, rows near zero sum
                m = (m + m.T).astype(np.float32) + np.eye(n, dtype=np.float32) * np.abs(m).sum()
            rows = [np.array(m[i], dtype=np.float32, copy=True) for i in range(n)]
            ptrs = (C.POINTER(C.c_float) * n)(*[r.ctypes.data_as(C.POINTER(C.c_float)) for r in rows])
            cof(ptrs, C.c_float(n))
            ref = np.array(rows)
            mine = np.zeros((MAXC, MAXC), np.float32)
            mine[:n, :n] = m
            L.or_circuit_inverse(mine.ctypes.data_as(C.POINTER(C.c_float)), n)
            assert np.array_equal(mine[:n, :n].view(np.uint32), ref.view(np.uint32)), (n, trial)


def test_laplace_charges_follow_cond_sigma_lap():
    s = hpic.Setup(circuit_deck(circuits=CIRCUITS), seed=5)
    info = s.info
    nc, G, ngx, ngy = info.cond_numr, info.Gsize, info.ngx, info.ngy
    lap = s.table("lap").reshape(nc, G)
    face, bnd, cid = s.table("face"), s.table("boundary"), s.table("cond_id")
    area = s.table("area")
    eps = (8.8542e-12 * s.table("eps_r").astype(np.float64)).astype(np.float32)
    dx, dy = float(np.float32(info.dx)), float(np.float32(info.dy))
    want = np.zeros((nc, nc), np.float32)
    for k in range(nc):
        P = lap[k]
        for n in range(G):
            if not cid[n]:
                continue
            sig = np.float32(0)
            if bnd[n] in (1, 3) and face[n] != 8:
                x, y = divmod(n, ngy)
                eT = x * (ngy - 1) + y
                eL = eT - ngy + 1 if x else eT
                eD = eT - 1 if y else eT
                eX = eL + eD - eT
                xo, yo = (ngy - 1 if x == ngx - 1 else 0), (1 if y == ngy - 1 else 0)
                eT, eL, eD = eT - xo - yo, eL - yo, eD - xo
                pL, pR = (n - ngy if x else n), (n if x == ngx - 1 else n + ngy)
                pD, pU = (n - 1 if y else n), (n if y == ngy - 1 else n + 1)

                def term(a, b, p, h):  # 0.5 * (eps_a + eps_b) * (P[n] - P[p]) / h, in double
                    return 0.5 * float(np.float32(eps[a] + eps[b])) * float(np.float32(P[n] - P[p])) / h

                up, down = lambda: term(eT, eL, pU, dy), lambda: term(eD, eX, pD, dy)
                left, right = lambda: term(eL, eX, pL, dx), lambda: term(eT, eD, pR, dx)
                v = {2: up, 3: down, 0: left, 1: right, 4: lambda: up() + left(), 5: lambda: up() + right(),
                     6: lambda: down() + left(), 7: lambda: down() + right()}[int(face[n])]()
                sig = np.float32(v)
            want[k, cid[n] - 1] = np.float32(want[k, cid[n] - 1] + np.float32(sig * area[n]))
    got = s.table("circuit")[5 * nc:].reshape(nc, nc)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    # a capacitance matrix: own charge positive, induced charges negative, rows near zero sum
    assert (np.diag(got) > 0).all() and (got - np.diag(np.diag(got)) <= 0).all()
    assert np.abs(got.sum(axis=1)).max() < 0.05 * np.diag(got).min()


def _transcribed_step(nc, cc, lapsig, vt, qconv, surf, pois_new, q, phi, pois, mode):
    """Efield_cuda's loops (src/cuda_Field.cu:49-80) line by line in float32
    (mode 0), and the charge balance (mode 1); lapsig[k, i] is Lap_SIG_Sol."""
    f = np.float32
    AM = np.zeros((nc, nc), f)
    b = np.zeros(nc, f)
    Kc = np.zeros(nc, f)
    S = np.zeros(nc, f)
    for i in range(nc):
        if mode == 1:
            acc = f(0)
            for j in range(nc):
                acc = f(acc + f(lapsig[j, i] * phi[j]))
            S[i] = f(acc + pois[i])
        else:
            S[i] = surf[i]
    K_t = f(0)
    for i in range(nc):
        a = cc[i]
        K_t = f(f(f(f(f(a[1] * q[0, i]) + f(a[2] * q[1, i])) + f(a[3] * q[2, i])) + f(a[4] * q[3, i])) / a[0])
        Kc[i] = K_t
        lead = f(f(vt[i] / a[0]) - K_t) if mode == 1 else f(f(vt[i] - K_t) / a[0])
        b[i] = f(f(f(f(lead - q[0, i]) - qconv[i]) + S[i]) - pois_new[i])
        for j in range(nc):
            AM[i, j] = f(lapsig[j, i] + f(f(1) / a[0])) if i == j else lapsig[j, i]
    L = oracle.lib()
    L.or_circuit_inverse.argtypes = [C.POINTER(C.c_float), C.c_int]
    inv = np.zeros((MAXC, MAXC), np.float32)
    inv[:nc, :nc] = AM
    L.or_circuit_inverse(inv.ctypes.data_as(C.POINTER(C.c_float)), nc)
    phi_new = np.zeros(nc, f)
    qn = q.copy()
    for i in range(nc):
        p = f(0)
        for j in range(nc):
            p = f(p + f(inv[i, j] * b[j]))
        phi_new[i] = p
        qn[3, i], qn[2, i], qn[1, i] = q[2, i], q[1, i], q[0, i]
        qn[0, i] = f(f(f(vt[i] - p) / cc[i][0]) - (Kc[i] if mode == 1 else K_t))
    return qn, phi_new


@pytest.mark.parametrize("mode", [0, 1])
def test_one_step_matches_the_transcription(mode):
    L = oracle.lib()
    fp = C.POINTER(C.c_float)
    L.or_circuit_step.argtypes = [C.c_int, fp, fp, fp, fp, fp, fp, fp, fp, fp, C.c_int]
    s = hpic.Setup(circuit_deck(), seed=5)
    nc = s.info.cond_numr
    tab = s.table("circuit")
    cc = tab[: 5 * nc].reshape(nc, 5).astype(np.float32)
    lapsig = tab[5 * nc:].reshape(nc, nc).astype(np.float32)
    lap4 = np.zeros(MAXC * MAXC, np.float32)
    for j in range(nc):
        lap4[j * MAXC: j * MAXC + nc] = lapsig[j]
    rng = np.random.default_rng(7 + mode)
    q = np.zeros((4, MAXC), np.float32)
    phi = np.zeros(MAXC, np.float32)
    pois = np.zeros(MAXC, np.float32)
    for step in range(40):
        vt = np.zeros(MAXC, np.float32)
        vt[0] = np.float32(200.0 * np.sin(0.0157 * step))
        qconv = np.zeros(MAXC, np.float32)
        qconv[:nc] = rng.normal(0, 1e-11, nc)
        surf = np.zeros(MAXC, np.float32)
        surf[:nc] = rng.normal(0, 1e-10, nc)
        pnew = np.zeros(MAXC, np.float32)
        pnew[:nc] = rng.normal(0, 1e-10, nc)
        want_q, want_phi = _transcribed_step(nc, cc, lapsig, vt, qconv, surf, pnew, q[:, :nc], phi[:nc], pois[:nc],
                                             mode)
        qq = q.copy()
        L.or_circuit_step(nc, cc.reshape(-1).ctypes.data_as(fp), lap4.ctypes.data_as(fp), vt.ctypes.data_as(fp),
                          qconv.ctypes.data_as(fp), surf.ctypes.data_as(fp), pnew.ctypes.data_as(fp),
                          qq.ctypes.data_as(fp), phi.ctypes.data_as(fp), pois.ctypes.data_as(fp), mode)
        assert np.array_equal(qq[:, :nc].view(np.uint32), want_q.view(np.uint32)), step
        assert np.array_equal(phi[:nc].view(np.uint32), want_phi.view(np.uint32)), step
        assert np.array_equal(pois[:nc], pnew[:nc])
        q = qq


def test_oracle_keeps_the_reference_quirks_and_mode_1_balances_charge():
    """Mode 0 (the reference) barely moves the driven electrode: its history
    term is the last conductor's, and (V - K_t) / cc0 mixes a voltage with a
    charge.  Mode 1 drives it through the R-L-C to the order of the source."""
    amp = {}
    for mode in (0, 1):
        s = hpic.Setup(circuit_deck(), seed=5)
        o = oracle.Oracle(s.table, s.info, hpic.default_opts(seed=5, circuit_mode=mode), 32)
        for sp in range(s.info.nsp):
            counts, arrs = s.particles(sp, layout=0)
            o.set_particles(sp, counts, *arrs)
        o.DepositBasic()
        top = 0.0
        for k in range(6):
            o.run(k * 25, 25)
            g = o.grid("CIRCUIT")
            assert np.isfinite(g).all()
            top = max(top, float(np.abs(g[5 * MAXC])))  # the driven electrode's potential
        amp[mode] = top
    assert amp[0] < 1.0 and amp[1] > 50.0, amp


def test_circuit_mode_is_checked():
    with pytest.raises(hpic.HpicError):
        hpic.Case(deck=circuit_deck(), seed=3, circuit_mode=2)


def _run_pair(deck, seed, steps, mode, batch_with=None):
    setup = hpic.Setup(deck, seed=seed)
    case = hpic.Case(setup=setup, seed=seed, circuit_mode=mode)
    o = oracle.Oracle(setup.table, setup.info, case.opts, 32, pcg_cluster=case.info.pcg_cluster,
                      pcg_block=case.info.pcg_block)
    for s in range(setup.info.nsp):
        counts, arrs = setup.particles(s, layout=0)
        o.set_particles(s, counts, *arrs)
    o.DepositBasic()
    if batch_with is not None:
        other = hpic.Case(deck=batch_with, seed=seed + 1)
        b = hpic.Batch([other, case])
        b.step(steps)
        b.close()
        other.close()
    else:
        case.step(steps)
    o.run(0, steps)
    return case, o


def _same(case, o):
    assert np.array_equal(case.grid("CIRCUIT").view(np.uint32), o.grid("CIRCUIT").view(np.uint32))
    assert np.array_equal(case.grid("PHI").view(np.uint32), o.grid("PHI").view(np.uint32))
    for s in range(case.info.nsp):
        gc, ga = case.particles(s)
        oc, oa = o.particles(s)
        assert np.array_equal(gc, oc)
        for a, b in zip(ga, oa):
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1])
def test_circuit_deck_bit_exact(mode):
    case, o = _run_pair(circuit_deck(), 21, 40, mode)
    assert case.status() == 0
    _same(case, o)
    assert np.abs(case.grid("CIRCUIT")[5 * MAXC: 5 * MAXC + 3]).max() > 0


@pytest.mark.gpu
def test_circuit_case_in_a_batch_equals_the_oracle():
    case, o = _run_pair(circuit_deck(), 22, 30, 1, batch_with=block_deck())
    _same(case, o)


@pytest.mark.gpu
def test_circuit_state_through_a_checkpoint(tmp_path):
    deck = circuit_deck()
    a = hpic.Case(deck=deck, seed=23, circuit_mode=1)
    a.step(20)
    path = str(tmp_path / "c.dump")
    a.save(path)
    a.step(15)
    b = hpic.Case(deck=deck, seed=23, circuit_mode=1)
    b.load(path)
    b.step(15)
    assert np.array_equal(a.grid("CIRCUIT").view(np.uint32), b.grid("CIRCUIT").view(np.uint32))
    assert np.array_equal(a.grid("PHI").view(np.uint32), b.grid("PHI").view(np.uint32))
