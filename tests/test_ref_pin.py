"""The oracle against the reference's own CUDA step code.

`make -C oracle ref_kernels` compiles the reference's src/cuda_Move.cu,
cuda_Sortboundary.cu, cuda_Deposit.cu, cuda_Field.cu, cuda_mcc.cu,
cuda_mccAr.cu, cuda_mccO2.cu, cuda_mccArO2.cu, cuda_Diagnostic.cu and
cuda_Fluid.cu as they are, for sm_100a
with the reference's own flags (-use_fast_math -rdc=true), into
oracle/_ref/libref_kernels.so; oracle/refk.py runs its kernels on states these
tests build from the oracle's.  The product kernels are compared with the
oracle bit for bit elsewhere; here the oracle itself is compared with the
reference's code, which pins the restatement:

* MoveE_Basic (src/cuda_Move.cu:181-270) vs the oracle's Move in move_mode 0
  (the reference's single wrap), then the oracle's SortBoundary vs the rules
  of SortBoundary_Basic (src/cuda_Sortboundary.cu:41-258) applied to the
  reference's Move output (sortboundary_np: that kernel raised
  cudaErrorInvalidAddressSpace on a B200 and is not launched);
* DepositAtom + DepositBoundary + SumSource (src/cuda_Deposit.cu:35-104,
  277-325) vs the oracle's Deposit_Basic;
* Cond_Sigma + VtoEfield (src/cuda_Field.cu:500-558,698-846) vs the oracle's
  field assembly on the same potential;
* PCG_float (src/cuda_Field.cu:942-1072) on the reference's own CSR matrix,
  launched on one warp, vs the oracle's field_mode 0 solve and an FP64 direct
  solve (its own launch races between the direction update and the next
  product: measured and reported, not compared);
* Argon/O2/ArO2_CrossSection and dev_anewvel / dev_newvel_IONSC /
  dev_maxwellv (src/cuda_mcc.cu:139-201) vs the oracle's lookup and
  kinematics on the same inputs;
* MCC_Ar_Basic (src/cuda_mcc.cu:97-106, src/cuda_mccAr.cu:41-232) vs the
  oracle's Ar MCC, both drawing the same scripted uniforms per cell (the
  reference's curand_uniform calls are routed to the lists by
  oracle/ref_shim.h), so every collision is compared one for one; the two
  draws passed to one kinematics call are taken left to right on both sides;
* Argon_Update_Source, Oxygen_Update_Source and ArO2_Update_Source
  (src/cuda_Diagnostic.cu:634-743) vs the oracle's fluid sources
  (include/hp_fluid.h) on the same averaged rates and densities;
* the Ar/O2 and O2 species handlers (src/cuda_mccArO2.cu:51-1129,
  src/cuda_mccO2.cu:2-866) vs the oracle's ladders, one collision per
  (species, target, energy, draws): this is what checks the channel tables.
  Electron collisions below the threshold of their ladder's first channel
  are skipped: there the reference adds the next cross section to a running
  sum it has not set (accumulator_undefined).

Timing.  MoveE_Basic, the Deposit kernels and PCG_float are also timed
against this library's kernels at the benchmark sizes (CUDA events, the
reference's launch shape), with the times printed.

Tolerances.  Integers are exact: cell counts, mover cell offsets, reaction
channels, conductor counts, created particles.  The reference is built with
-use_fast_math (approximate exp/log/pow/sin/cos/tan, contracted multiply-
adds) and adds charge with float atomics in arrival order, while the oracle
uses correctly rounded functions and FP64 sums, so floating-point results
agree within the bounds stated at each assertion.
"""
import numpy as np
import pytest

import hpic
import oracle
import refk
from hpic.decks import ccp_deck

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refk.available(),
                                 reason="oracle/_ref/libref_kernels.so not built (no reference tree where build() ran)")]

MPNC = 512  # slots per node in the reference layout: 9x the largest cell


def oracle_for(deck, seed, **kw):
    kw.setdefault("move_mode", 0)
    kw.setdefault("field_mode", 0)
    S = hpic.Setup(deck, seed=seed, **kw)
    o = oracle.Oracle(S.table, S.info, S.opts, 32)
    for s in range(S.info.nsp):
        counts, arrs = S.particles(s, layout=0)
        o.set_particles(s, counts, *arrs)
    return S, o


def rel_err(a, b, scale):
    return float(np.max(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)), initial=0.0) / scale)


# ------------------------------------------------------------ Move + Sort
NEUMANN = {  # StructureIndex code -> (node shift in units of (ngy, 1), flip x, flip y) (src/cuda_Sortboundary.cu:213-236)
    -2: ((1, 0), True, False), -6: ((-1, 0), True, False), -4: ((0, 1), False, True), -8: ((0, -1), False, True),
    -12: ((1, 1), True, True), -16: ((-1, 1), True, True), -20: ((1, -1), True, True), -24: ((-1, -1), True, True),
}


def sortboundary_np(S, st):
    """SortBoundary_Basic (src/cuda_Sortboundary.cu:41-258) for decks with no
    dielectric, on the reference layout after MoveE_Basic: each mover goes to
    the cell its offset names, or is reflected (Neumann codes), counted on a
    conductor (codes >= 100) or absorbed (-1 and the codes the reference
    leaves undefined).  Returns per species (counts per cell, arrays) with the
    movers appended after each cell's stayers, and the conductor counts."""
    info = S.info
    ngy, ncy, G = info.ngy, info.ncy, info.Gsize
    sidx = S.table("sidx").reshape(info.ncx + 2, ncy + 2)
    cond = np.zeros(info.nsp * info.cond_numr, np.float32)
    out = []
    for s in range(info.nsp):
        counts, arrs = refk.from_ref(st, s)
        lists = [[] for _ in range(info.Csize)]
        mc, ma, mcell = refk.movers_from_ref(st, s)
        src = np.repeat(np.arange(info.Csize), mc)
        for q in range(src.size):
            i, j = divmod(int(src[q]), ncy)
            m = int(mcell[q])
            di = int(np.sign(m)) if abs(m) > 1 else 0
            dj = m - di * ngy
            code = int(sidx[i + 1 + di, j + 1 + dj])
            x, y, vx, vy, vz = (ma[k][q] for k in range(5))
            if code == 0:
                ti, tj = i + di, j + dj
            elif code in NEUMANN:
                (si, sj), fx, fy = NEUMANN[code]
                ti, tj = i + di + si, j + dj + sj
                if fx:
                    x, vx = np.float32(1) - x, -vx
                if fy:
                    y, vy = np.float32(1) - y, -vy
            else:
                if code >= 100:
                    cond[s * info.cond_numr + code - 101] += 1
                continue
            lists[ti * ncy + tj].append((x, y, vx, vy, vz))
        start = np.concatenate([[0], np.cumsum(counts)])
        new_counts = counts.copy()
        cols = [[] for _ in range(5)]
        for c in range(info.Csize):
            for k in range(5):
                cols[k].extend(arrs[k][start[c]:start[c + 1]].tolist())
                cols[k].extend(p[k] for p in lists[c])
            new_counts[c] += len(lists[c])
        out.append((new_counts, [np.asarray(v, np.float32) for v in cols]))
    return out, cond


@pytest.mark.parametrize("name,deck,seed", [
    ("ar_65x33", ccp_deck(65, 33, 0.02, 0.01, ppc=30), 99),
    ("ar_33x17_hv", ccp_deck(33, 17, 0.01, 0.005, ppc=20, pressure_torr=0.1, voltage=300.0), 777),
])
def test_move_sort_match_reference(name, deck, seed):
    S, o = oracle_for(deck, seed)
    info = S.info
    o.DepositBasic()
    o.Field(1)
    ex, ey = o.grid("EX"), o.grid("EY")
    st = refk.to_ref(info, MPNC, [o.particles(s) for s in range(info.nsp)])
    rc = refk.case_from_oracle(o, MPNC)
    refk.move(rc, st, ex, ey)
    o.Move()
    for s in range(info.nsp):
        # stayers: same cells, same order
        rc_cnt, ra = refk.from_ref(st, s)
        oc, oa = o.particles(s)
        assert np.array_equal(rc_cnt, oc), f"{name} species {s}: stayers per cell differ"
        vscale = max(float(np.abs(oa[2]).max()), float(np.abs(oa[3]).max()))
        assert rel_err(ra[0], oa[0], 1.0) <= 1e-6 and rel_err(ra[1], oa[1], 1.0) <= 1e-6, "stayer offsets"
        for q in (2, 3):
            assert rel_err(ra[q], oa[q], vscale) <= 1e-6, f"stayer velocities ({name}, species {s})"
        assert np.array_equal(ra[4], oa[4]), "vz is copied"
        # movers: same count per cell, in the same order; where the cell
        # entered is plasma the destination is the crossing itself (the
        # oracle applies wall rules in Move, the reference in SortBoundary)
        mc, ma, mcell = refk.movers_from_ref(st, s)
        om, _, ocodes = o.movers(s)
        assert np.array_equal(mc, om), f"{name} species {s}: movers per cell differ"
        di = np.where(np.abs(mcell) > 1, np.sign(mcell), 0)
        dj = mcell - di * info.ngy
        assert (np.abs(dj) <= 1).all()
        src = np.repeat(np.arange(info.Csize), mc)
        si, sj = src // info.ncy, src % info.ncy
        sidx = S.table("sidx").reshape(info.ncx + 2, info.ncy + 2)
        plasma = sidx[si + 1 + di, sj + 1 + dj] == 0
        assert np.array_equal(((di + 1) * 3 + dj + 1)[plasma], ocodes[plasma].astype(np.int64)), "mover cell offsets"
    # SortBoundary_Basic raised cudaErrorInvalidAddressSpace on a B200 on this
    # state although a read-only device replay of its index arithmetic found
    # every index in range (refk.sort_probe); it is not launched here.  Its
    # rules are applied by sortboundary_np to the reference's Move output.
    cells, cond = sortboundary_np(S, st)
    o.SortBoundary()
    occ, _, _ = o.counters()
    assert np.array_equal(cond, occ), f"{name}: conductor counts {cond} vs {occ}"
    for s in range(info.nsp):
        rc_cnt, ra = cells[s]
        oc, oa = o.particles(s)
        assert np.array_equal(rc_cnt, oc), f"{name} species {s}: particles per cell after SortBoundary"
        # compare each cell as a set (the reference re-bins with atomics, in
        # arrival order), ordered by vz, which no step of Move or Sort changes
        cell = np.repeat(np.arange(info.Csize), oc)
        ro = np.lexsort((ra[4], cell))
        oo = np.lexsort((oa[4], cell))
        assert np.array_equal(ra[4][ro], oa[4][oo])
        vscale = max(float(np.abs(oa[2]).max()), float(np.abs(oa[3]).max()))
        for q in range(4):
            scale = 1.0 if q < 2 else vscale
            err = rel_err(ra[q][ro], oa[q][oo], scale)
            assert err <= 1e-6, f"{name} species {s} array {q}: {err:.2e}"


# ------------------------------------------------------------ Deposit
def test_deposit_matches_reference():
    S, o = oracle_for(ccp_deck(65, 33, 0.02, 0.01, ppc=30), 99)
    info = S.info
    o.DepositBasic()
    st = refk.to_ref(info, MPNC, [o.particles(s) for s in range(info.nsp)])
    rc = refk.case_from_oracle(o, MPNC)
    den, src, _ = refk.deposit(rc, st, S.table("face"), S.table("boundary"), S.table("cond_id"), S.table("area"))
    oden, osrc = o.grid("DEN"), o.grid("SOURCE")
    G = info.Gsize
    for s in range(info.nsp):
        d, od = den[s * G:(s + 1) * G], oden[s * G:(s + 1) * G]
        # float atomics over <= 4 x 60 weights per node: <= 1e-5 of the largest node
        assert rel_err(d, od, float(np.abs(od).max())) <= 1e-5
    qs = max(abs(rc.q_density[s]) * float(np.abs(oden[s * G:(s + 1) * G]).max()) for s in range(info.nsp)) / 8.8542e-12
    assert rel_err(src, osrc, qs) <= 1e-5


# ------------------------------------------------------------ Efield
def test_efield_matches_reference():
    S, o = oracle_for(ccp_deck(65, 33, 0.02, 0.01, ppc=30, voltage=200.0), 99)
    info = S.info
    o.DepositBasic()
    o.Field(37)
    phi, ex0, ey0 = o.grid("PHI"), o.grid("EX"), o.grid("EY")
    rc = refk.case_from_oracle(o, 4)
    c = o.c
    geom = [c.dx, c.dy, c.hdx, c.hdy, c.idx, c.idy, c.idxy]
    eps = o.keep["eps"]
    ex, ey, _ = refk.efield(rc, geom, S.table("face"), S.table("boundary"), eps, o.grid("DEN"),
                            np.zeros(info.Gsize, np.float32), phi)
    es = max(float(np.abs(ex0).max()), float(np.abs(ey0).max()))
    assert rel_err(ex, ex0, es) <= 1e-5 and rel_err(ey, ey0, es) <= 1e-5


# ------------------------------------------------------------ PCG
def test_pcg_matches_reference():
    S, o = oracle_for(ccp_deck(129, 65, 0.04, 0.02, ppc=20), 5)
    o.DepositBasic()
    b_node = o.grid("B")
    o.Field(1)
    idx = S.table("a_idx")
    unk = np.nonzero(idx)[0]
    n = int(idx.max())
    b = np.zeros(n, np.float32)
    b[idx[unk] - 1] = b_node[unk]
    ai, aj, val, m = S.table("ai"), S.table("aj"), S.table("a_val"), S.table("matm")
    tol2 = float(o.c.pcg_tol2)
    _, _, it_or = o.counters()
    # the FP64 solution of the reference's own CSR system
    import scipy.sparse as sps
    import scipy.sparse.linalg as spl
    A = sps.csr_matrix((val.astype(np.float64), aj - 1, ai - 1), shape=(n, n))
    xd = spl.spsolve(A.tocsc(), b.astype(np.float64))
    xs = float(np.abs(xd).max())
    xo = np.zeros(n, np.float64)
    xo[idx[unk] - 1] = o.grid("PHI_POIS")[unk]
    # PCG_float on one warp (its direction update and the next product do not
    # race there): the same solver as the oracle's field_mode 0
    x1, it1, ms1 = refk.pcg(ai, aj, val, m, b, np.zeros(n, np.float32), tol2, nblocks=1, nthreads=32)
    # and as the reference launches it, which races on a B200 (measured, see
    # the design notes): reported, not compared
    x0, it0, ms0 = refk.pcg(ai, aj, val, m, b, np.zeros(n, np.float32), tol2)
    print(f"PCG_float one warp: {it1} it, {ms1:.2f} ms, |x-x64| {rel_err(x1, xd, xs):.2e}; "
          f"reference launch: {it0} it, {ms0:.2f} ms, |x-x64| {rel_err(x0, xd, xs):.2e}; "
          f"oracle: {it_or[0]} it, |x-x64| {rel_err(xo, xd, xs):.2e}")
    # the same absolute r'z rule stops both: iterations within 5 % and the
    # same solution to the solver's accuracy (1e-2 of the largest potential)
    assert abs(it1 - it_or[0]) <= max(3, 0.05 * it_or[0]), (it1, it_or[0])
    assert rel_err(x1, xd, xs) <= 1e-2 and rel_err(xo, xd, xs) <= 1e-2
    assert rel_err(x1, xo, xs) <= 1e-2


TIMED_CASES = {  # the benchmark cases: CPU-sized Ar, the headline Ar case, Ar/O2 80/20
    "ar_129x65_50ppc": dict(ngx=129, ngy=65, xlen=0.04, ylen=0.02, ppc=50, voltage=100.0, pressure_torr=0.05),
    "ar_513x257_200ppc": dict(ngx=513, ngy=257, xlen=0.16, ylen=0.08, ppc=200, voltage=100.0, pressure_torr=0.05),
    "aro2_257x129_100ppc": dict(ngx=257, ngy=129, xlen=0.08, ylen=0.04, ppc=100, voltage=200.0, pressure_torr=0.1,
                                gas="ArO2", te_ev=3.0, aro2_ratio=(80, 20),
                                ion_density={"Ar+": 1e15, "O2+": 2e14, "O+": 0.0, "O-": 2e14}),
}


@pytest.mark.parametrize("name", list(TIMED_CASES))
def test_move_and_deposit_time_against_the_reference_kernels(name):
    """The benchmark cases: Ar 129x65 at 50 particles per cell and species,
    Ar 513x257 at 200 (52M particles, 100 V, 50 mTorr) and 80/20 Ar/O2
    257x129 at 100 (five species, 200 V, 100 mTorr).  On the initial state
    and the field of the first step, the reference's MoveE_Basic and its Deposit kernels
    (DepositInitDensity, DepositAtom, DepositBoundary, SumSource) are timed
    with CUDA events over 5 launches on restored inputs, with the launch
    shape the reference picks (src/cuda_Init.cu:35-46); this library's
    kernels are timed per launch over three op-by-op steps of the same case
    (hp_profile_step).  Both sides' times are printed.  The reference's Move
    and this library's Move (move_mode 0, its one-crossing rule) leave the
    same stayers in each cell, but for cells where the two builds round a
    position at a cell edge differently (fast-math contractions against
    explicit fused multiply-adds): at most 1e-4 of the cells, or 2."""
    w = dict(TIMED_CASES[name])
    deck = ccp_deck(w.pop("ngx"), w.pop("ngy"), w.pop("xlen"), w.pop("ylen"), **w)
    S = hpic.Setup(deck, seed=11, move_mode=0, field_mode=2)
    info = S.info
    o = oracle.Oracle(S.table, S.info, S.opts, 32)  # the float constants of the reference case
    rc = refk.case_from_oracle(o, MPNC)
    del o
    st = refk.to_ref(info, MPNC, [S.particles(s, layout=0) for s in range(info.nsp)])
    case = hpic.Case(setup=S, seed=11, move_mode=0, field_mode=2)
    case.Deposit()
    case.set_tstep(1)
    case.Field()
    ex, ey = case.grid("EX"), case.grid("EY")
    try:
        refk.set_timing(5)
        refk.deposit(rc, st, S.table("face"), S.table("boundary"), S.table("cond_id"), S.table("area"))
        dep_ref = refk.last_ms()[:4]
        refk.move(rc, st, ex, ey)
        move_ref = refk.last_ms()[0]
    finally:
        refk.set_timing(0)
    case.Move()
    G = info.Gsize
    node = refk.cell_to_node(info)
    for s in range(info.nsp):
        ours, _ = case.particles(s)
        ref = st.pnc[s * G + node]
        differ = int(np.count_nonzero(ours != ref))
        assert differ <= max(1e-4 * info.Csize, 2), f"species {s}: stayers differ in {differ} of {info.Csize} cells"
        assert abs(int(ours.sum()) - int(ref.sum())) <= 1e-6 * int(ref.sum()) + 8
    case.SortBoundary()
    case.MCC()
    case.Deposit()
    stats = {k: ms / max(n, 1) for k, n, ms in case.profile(3)}
    case.close()
    ours_dep = sum(stats.get(k, 0.0) for k in ("k_deposit_cells", "k_deposit_nodes", "k_source"))
    ours_sort = stats.get("k_sort_count", 0.0) + stats.get("k_sort_push", 0.0)
    print(f"{name} ({info.nsp} species), {int(st.pnc.sum())} stayers after the reference Move: "
          f"MoveE_Basic {move_ref:.3f} ms; DepositInitDensity/Atom/Boundary/SumSource "
          f"{' / '.join(f'{t:.3f}' for t in dep_ref)} = {sum(dep_ref):.3f} ms | this library: k_move "
          f"{stats['k_move']:.3f} ms (+ sort {ours_sort:.3f} ms, the boundary rules the reference applies in "
          f"SortBoundary), deposit {ours_dep:.3f} ms")
    assert move_ref > 0 and min(dep_ref) > 0 and stats["k_move"] > 0 and ours_dep > 0


@pytest.mark.parametrize("ngx,ngy,xl,yl", [(129, 65, 0.04, 0.02), (513, 257, 0.16, 0.08)])
def test_pcg_solve_time_against_the_reference_kernel(ngx, ngy, xl, yl):
    """The first Poisson solve of a CCP deck (warm start 0, the reference's
    absolute r'z rule, field mode 0): this library's PCG (one cluster, or the
    whole-GPU cooperative solve above 65,536 nodes) against the reference's
    PCG_float launched as PCG_SOLVER launches it, on the same right-hand
    side, both timed with CUDA events.  This library's solve must take less
    time; both per-iteration times are printed."""
    deck = ccp_deck(ngx, ngy, xl, yl, ppc=4, max_np_factor=8)
    S, o = oracle_for(deck, 5)
    o.DepositBasic()
    b_node = o.grid("B")
    idx = S.table("a_idx")
    unk = np.nonzero(idx)[0]
    n = int(idx.max())
    b = np.zeros(n, np.float32)
    b[idx[unk] - 1] = b_node[unk]
    ai, aj, val, m = S.table("ai"), S.table("aj"), S.table("a_val"), S.table("matm")
    tol2 = float(o.c.pcg_tol2)
    refk.pcg(ai, aj, val, m, b, np.zeros(n, np.float32), tol2)  # warm-up (module load, first launch)
    _, it_ref, ms_ref = refk.pcg(ai, aj, val, m, b, np.zeros(n, np.float32), tol2)
    case = hpic.Case(setup=S, seed=5, field_mode=0, move_mode=0)
    case.set_tstep(1)
    case.Field()  # warm-up of the launch path (the solve starts from 0 again below)
    case.set_grid("PCG_X", np.zeros(case.info.Gsize, np.float32))
    case.set_tstep(0)
    # one profiled step: its Field phase solves the same system from 0 (the
    # Poisson part holds the conductors at 0 V, whatever the step's voltage)
    stats = {name: ms for name, _, ms in case.profile(1)}
    it_ours = case.pcg_iters()[0]
    ms_ours = stats.get("k_pcg", stats.get("k_pcg_grid"))
    print(f"{ngx}x{ngy}: PCG_float (reference launch) {it_ref} it {ms_ref:.3f} ms = {1e3 * ms_ref / max(it_ref, 1):.2f} "
          f"us/it; this library ({'grid' if 'k_pcg_grid' in stats else 'cluster'} {case.info.pcg_cluster} CTAs) "
          f"{it_ours} it {ms_ours:.3f} ms = {1e3 * ms_ours / max(it_ours, 1):.2f} us/it")
    assert ms_ours < ms_ref


# ------------------------------------------------------------ cross sections, kinematics
@pytest.mark.parametrize("gas_name,gas", [("Ar", 0), ("O2", 1), ("ArO2", 2)])
def test_cross_sections_match_reference(gas_name, gas):
    deck = ccp_deck(17, 9, 0.005, 0.0025, ppc=2, gas=gas_name)
    S, o = oracle_for(deck, 3)
    sc = S.table("scalars")
    n_logx, idlogx = int(sc[14]), float(sc[15])
    tab = S.table("xsec")
    width = tab.size // n_logx
    t = tab.reshape(n_logx, width)
    rng = np.random.default_rng(7)
    engy = np.concatenate([10 ** rng.uniform(-3, 4.5, 4000), 10 ** np.linspace(-3, 4.5, 400)]).astype(np.float32)
    # the table rows the lookup interpolates between
    row = np.clip(np.floor(idlogx * (np.log10(engy.astype(np.float64)) - t[0, 0])).astype(int), 0, n_logx - 2)
    worst = 0.0
    for ch in range(width - 2):
        r = refk.xsec(gas, ch, n_logx, idlogx, tab, width, engy).astype(np.float64)
        q = o.xsec(ch, engy).astype(np.float64)
        assert np.array_equal(r == 0, q == 0), f"channel {ch}: zero entries differ"
        # the reference's fast-math log10 moves the interpolation coordinate by
        # a few 1e-6: within 1e-4 of the larger of the value and the two table
        # entries it lies between
        scale = np.maximum(np.abs(q), np.maximum(np.abs(t[row, 2 + ch]), np.abs(t[row + 1, 2 + ch])))
        e = float(np.max(np.abs(r - q) / np.where(scale > 0, scale, 1.0)))
        worst = max(worst, e)
        assert e <= 1e-4, f"{gas_name} channel {ch}: {e:.2e} of the local table scale"
    print(f"{gas_name}: {width - 2} channels, worst difference {worst:.2e} of the local table scale")


def test_kinematics_match_reference():
    S, o = oracle_for(ccp_deck(17, 9, 0.005, 0.0025, ppc=2), 3)
    rng = np.random.default_rng(11)
    n = 20000
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    u1, u2 = rng.uniform(1e-7, 1.0, n), rng.uniform(1e-7, 1.0, n)
    energy = 10 ** rng.uniform(-1, 3, n)
    vel = rng.uniform(1e5, 5e6, n)
    cases = {
        0: np.column_stack([energy, vel, d, u1, u2]),
        1: np.column_stack([d * vel[:, None], vel, u1, u2]),
        2: np.column_stack([rng.uniform(0, 3.3, n), rng.uniform(100, 1e6, n), u1, u2]),
    }
    for kind, inp in cases.items():
        inp = inp.astype(np.float32)
        r = refk.kinematics(kind, inp)
        q = o.kinematics(kind, inp)
        mag = np.linalg.norm(q.astype(np.float64), axis=1)
        err = np.linalg.norm(r.astype(np.float64) - q, axis=1) / np.maximum(mag, 1e-30)
        print(f"kinematics {kind}: max {err.max():.2e}, 99.9% {np.quantile(err, 0.999):.2e}, median {np.median(err):.2e}")
        # fast-math pow/sin/cos: the new direction within 1e-3 for every draw, 1e-5 typically
        assert err.max() <= 1e-3 and np.median(err) <= 1e-5, kind


# ------------------------------------------------------------ MCC, Ar set
# Velocity tolerance of a collision: 2e-3 of the speed plus, for electrons,
# 1200 m/s.  The reference splits the ionisation energy as
# 10 tan(U atan(E/20)) with the fast-math __tanf, whose absolute error
# (~3.6e-7) leaves a created electron of a few micro-eV with no speed or a
# shortened one; 1200 m/s is the speed of 3.6e-6 eV.  anewvel's fast-math
# pow/sin/cos set the 2e-3 (small-angle scattering at low energy).
E_FLOOR = 1200.0


def ar_mcc_mismatch(S, o, st_ref, mccr, node):
    """None when the oracle reproduces the reference's MCC, else why not."""
    info = S.info
    _, omc, _ = o.counters()
    omc = omc.reshape(info.Csize, -1)
    if not np.array_equal(mccr[node][:, :7].astype(np.int64), omc[:, :7].astype(np.int64)):
        return "reaction tallies per cell"
    for s in range(info.nsp):
        rcnt, ra = refk.from_ref(st_ref, s)
        oc, oa = o.particles(s)
        if not np.array_equal(rcnt, oc):
            return f"species {s}: particles per cell"
        if not (np.array_equal(ra[0], oa[0]) and np.array_equal(ra[1], oa[1])):
            return f"species {s}: positions (copied in every collision)"
        v_r = np.stack(ra[2:5], 1).astype(np.float64)
        v_o = np.stack(oa[2:5], 1).astype(np.float64)
        dv = np.linalg.norm(v_r - v_o, axis=1)
        sp = np.linalg.norm(v_o, axis=1)
        bad = dv > 2e-3 * sp + (E_FLOOR if s == 0 else 0.0)
        rel = dv / np.maximum(sp, 1e-30)
        print(f"species {s}: {bad.sum()} of {sp.size} velocities outside; median relative {np.median(rel):.1e}")
        if bad.any():
            return f"species {s}: velocities"
    return None


def test_mcc_ar_matches_reference_with_the_same_draws():
    # 1 Torr and 12 eV electrons: many collisions per step in every channel;
    # draws skewed toward 0 make most particles collide
    deck = ccp_deck(33, 17, 0.01, 0.005, ppc=24, pressure_torr=1.0, voltage=200.0, te_ev=12.0)
    S, o = oracle_for(deck, 21)
    info = S.info
    rng = np.random.default_rng(5)
    species = [o.particles(s) for s in range(info.nsp)]
    counts = [sp[0] for sp in species]
    per_cell = 8 * counts[1] + (int(o.c.mcc_n) + 16) * counts[0] + 8
    start = np.concatenate([[0], np.cumsum(per_cell)]).astype(np.int64)
    u = rng.uniform(0, 1, start[-1]) ** rng.choice([1.0, 1.0, 6.0], start[-1])
    u = np.maximum(u, 1e-7).astype(np.float32)
    # the reference keys its lists by node, the oracle by cell
    node = refk.cell_to_node(info)
    rstart = np.zeros(info.Gsize + 1, np.int64)
    lens = np.zeros(info.Gsize, np.int64)
    lens[node] = per_cell
    rstart[1:] = np.cumsum(lens)
    ru = np.zeros(rstart[-1], np.float32)
    for cidx in range(info.Csize):
        ru[rstart[node[cidx]]:rstart[node[cidx] + 1]] = u[start[cidx]:start[cidx + 1]]
    st = refk.to_ref(info, MPNC, species)
    rc = refk.case_from_oracle(o, MPNC)
    sc = S.table("scalars")
    mcc = [sc[0], sc[1]]
    imcc = [int(sc[11]), int(sc[12]), int(sc[14]), info.n_reactions]
    fluid = S.table("fluid_den")[:info.Gsize]
    mccr, over = refk.mcc_ar(rc, st, mcc, imcc, sc[15], S.table("vsave"), S.table("xsec"), S.table("sigv"),
                             S.table("collf"), S.table("back_den1"), S.table("back_vel1"), fluid, ru, rstart)
    assert over == 0
    o.set_script(u, start)
    o.MCC(1)
    assert o.script_overrun() == 0
    _, omc, _ = o.counters()
    tallies = omc.reshape(info.Csize, -1)[:, :7].sum(axis=0)
    print("collisions per channel:", tallies)
    assert (tallies[[0, 1, 2, 3, 5, 6]] > 0).all(), "every Ar channel occurs"
    why = ar_mcc_mismatch(S, o, st, mccr, node)
    assert why is None, why
    # the comparison follows the draws one for one: taking the two draws of
    # every kinematics call in the other order no longer reproduces it
    S7, o7 = oracle_for(deck, 21)
    o7.set_script(u, start, pair_rl=7)
    o7.MCC(1)
    assert ar_mcc_mismatch(S7, o7, st, mccr, node) is not None


# ------------------------------------------------------------ MCC, oxygen sets
TARGETS = {  # targets of each species' collision check (src/cuda_mccArO2.cu:1143-1190, src/cuda_mccO2.cu:867-977)
    2: {0: 9, 1: 2, 2: 5, 3: 4, 4: 5},
    1: {0: 7, 1: 4, 2: 4, 3: 5},
}
# first reaction channel of each electron target's ladder, and one past its
# last (src/cuda_mccArO2.cu:91-435, src/cuda_mccO2.cu:2-429)
E_LADDER = {2: [0, 4, 5, 19, 27, 35, 36, 37, 44, 46], 1: [0, 14, 22, 30, 31, 32, 39, 41]}


def accumulator_undefined(gas, isp, t, engy, th):
    """True where the reference's electron ladder reads its running sum
    before setting it: the first channel is tested as
    `engy > Th && R1 <= (SumSigma = CS)`, so below that channel's threshold
    the next `SumSigma += CS` starts from the previous collider's sum (or an
    unset register).  The oracle, like the library, starts from 0."""
    if isp != 0:
        return False
    first, end = E_LADDER[gas][t], E_LADDER[gas][t + 1]
    return end - first >= 2 and not engy > th[first]


@pytest.mark.parametrize("gas_name,gas", [("ArO2", 2), ("O2", 1)])
def test_oxygen_ladders_match_reference(gas_name, gas):
    deck = ccp_deck(17, 9, 0.005, 0.0025, ppc=2, gas=gas_name)
    S, o = oracle_for(deck, 3, o2_all_species=1)
    info = S.info
    sc = S.table("scalars")
    tnrct = info.n_reactions
    imcc = [int(sc[12]), int(sc[14]), tnrct]
    spc = S.table("species").reshape(-1, 16)
    escale = [float(spc[s, 6]) for s in range(info.nsp)]
    bv1 = float(S.table("back_vel1")[info.ngy + 1])
    bv2 = float(S.table("back_vel2")[info.ngy + 1])
    rng = np.random.default_rng(13 + gas)
    n, nu = 6000, 24
    th = S.table("collf").reshape(-1, 4)[:, 2]
    hit = set()
    compared = skipped = 0
    worst = 0.0
    for isp, nt in TARGETS[gas].items():
        t = rng.integers(0, nt, n)
        engy = 10 ** rng.uniform(-2, 3, n)
        vmag = np.sqrt(engy / escale[isp])
        d = rng.normal(size=(n, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        v = (d * vmag[:, None]).astype(np.float32)
        u = (rng.uniform(0, 1, (n, nu)) ** rng.choice([1.0, 4.0, 12.0], (n, 1))).astype(np.float32)
        u = np.maximum(u, 1e-7)
        cnt, vout, mccr, over = refk.oxy_collide(gas, isp, imcc, sc[15], escale, S.table("vsave"), S.table("xsec"),
                                                 S.table("sigv"), S.table("collf"), v, t, np.full(n, bv1),
                                                 np.full(n, bv2), u)
        for k in range(n):
            e32 = np.float32(escale[isp]) * np.float32(np.dot(v[k].astype(np.float32), v[k].astype(np.float32)))
            if accumulator_undefined(gas, isp, int(t[k]), e32, th):
                skipped += 1
                continue
            compared += 1
            rch = np.nonzero(mccr[k])[0]
            assert rch.size <= 1
            ch, keep, vo, bsp, bv, kill, ov = o.collide_oxy(isp, int(t[k]), v[k], bv1, bv2, u[k])
            assert not ov
            assert (rch[0] if rch.size else -1) == ch, f"{gas_name} species {isp} target {t[k]} E={engy[k]:.3g}: channel"
            if ch >= 0:
                hit.add(ch)
            # expected particles per species: births in order, then the collider if it stays
            want = [[] for _ in range(info.nsp)]
            for q in range(2):
                if bsp[q] >= 0:
                    want[bsp[q]].append(bv[q])
            if keep:
                want[isp].append(vo)
            vin = float(np.linalg.norm(v[k]))
            for s in range(info.nsp):
                assert cnt[k, s] == len(want[s]), f"{gas_name} species {isp} channel {ch}: species {s} count"
                for q, w in enumerate(want[s]):
                    dv = float(np.linalg.norm(vout[k, s, q] - w))
                    worst = max(worst, dv / vin)
                    assert dv <= 2e-3 * vin + (E_FLOOR if s == 0 else 0.0), \
                        f"{gas_name} species {isp} channel {ch}: velocity {vout[k, s, q]} vs {w}"
    print(f"{gas_name}: {compared} collisions compared, {skipped} skipped (running sum undefined in the "
          f"reference), largest |dv|/|v_in| {worst:.1e}, channels hit {sorted(hit)}")
    assert len(hit) >= 0.5 * tnrct, f"{gas_name}: only {len(hit)} of {tnrct} channels exercised"


# ------------------------------------------------------------ fluid sources
@pytest.mark.parametrize("gas", ["Ar", "O2", "ArO2"])
def test_fluid_sources(gas):
    """The sources of the fluid species from averaged collision rates, node
    densities and the background gas: every channel the sources sum is given
    a rate of its own size, so a term added to the wrong species, with the
    wrong sign or factor, or read from the wrong channel shows.  The
    reference's kernels multiply and add in float as the restatement; its
    -use_fast_math contraction only meets the 2 x R terms, which are exact."""
    S = hpic.Setup(ccp_deck(17, 9, 0.005, 0.0025, gas=gas, ppc=4), seed=3)
    info = S.info
    g = {"Ar": 0, "O2": 1, "ArO2": 2}[gas]
    n, tnrct, nf = 4096, info.n_reactions, info.n_fluid
    rng = np.random.default_rng(11 + g)
    rr = S.table("collf").reshape(-1, 4)[:, 3].astype(np.float32)
    rates = (10 ** rng.uniform(18, 23, (n, tnrct)) * (rng.uniform(size=(n, tnrct)) > 0.1)).astype(np.float32)
    ave_e = (10 ** rng.uniform(13, 17, n)).astype(np.float32)
    fden = (10 ** rng.uniform(12, 19, (nf, n))).astype(np.float32)
    bd1 = np.full(n, S.table("back_den1").max(), np.float32) * rng.uniform(0.5, 1.5, n).astype(np.float32)
    bd2 = (bd1 * np.float32(0.25)).astype(np.float32) if g == 2 else np.zeros(n, np.float32)
    R_ref, S_ref = refk.fluid_source(g, info.ngy, rates, rr, ave_e, fden, bd1, bd2)
    eden = (0.25 * ave_e.astype(np.float64)).astype(np.float32)
    R_or, S_or = oracle.fluid_sources(g, rates, fden, eden, bd1, bd2, rr)
    assert np.array_equal(R_ref.view(np.uint32), R_or.view(np.uint32)), "neutral reaction rates"
    scale = np.maximum(np.abs(S_ref), 1.0)
    err = float(np.max(np.abs(S_ref.astype(np.float64) - S_or) / scale))
    print(f"{gas}: {nf} fluid species x {n} nodes, largest relative difference {err:.1e}")
    assert np.array_equal(S_ref.view(np.uint32), S_or.view(np.uint32)), f"sources differ (largest {err:.1e})"
