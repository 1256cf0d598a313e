"""ctypes binding of oracle/_ref/libref_kernels.so: the reference's own CUDA
step code (compiled from its sources by `make -C oracle ref_kernels`) run on
states the tests supply.  Test infrastructure only.

Layouts.  The oracle keeps a species' particles in cell order with a count
per cell (cell = i * ncy + j).  The reference keeps particle k of node
ID = i * ngy + j at ID + k * Gsize inside its species block of mpnc * Gsize
slots (src/cuda_Move.cu:195).  `to_ref` / `from_ref` convert between the two.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libref_kernels.so")

_F = C.POINTER(C.c_float)
_I = C.POINTER(C.c_int)
_LL = C.POINTER(C.c_longlong)


class RkCase(C.Structure):
    _fields_ = [("ngx", C.c_int), ("ngy", C.c_int), ("nsp", C.c_int), ("mpnc", C.c_int),
                ("dt_dx", C.c_float), ("dt_dy", C.c_float),
                ("ascale", C.c_float * 5), ("q_density", C.c_float * 5), ("escale", C.c_float * 5),
                ("np2c", C.c_float * 5)]


_lib = None


def available():
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB)
        P = C.POINTER(RkCase)
        sig = {
            "rk_last_error": (C.c_char_p, []),
            "rk_set_timing": (None, [C.c_int]),
            "rk_last_ms": (None, [_F]),
            "rk_move": (C.c_int, [P, _F, _F, _I, _I, _F, _F, _F, _F, _F, _I]),
            "rk_sortboundary": (C.c_int, [P, C.c_int, _I, _I, _I, _F, _F, _F, _F, _F, _I, _F, _I]),
            "rk_sort_probe": (C.c_int, [P, _I, _I, _I, _I, _LL, _I]),
            "rk_deposit": (C.c_int, [P, _I, _I, _I, _F, _I, _F, _F, _F, _F, _F, _F, _F]),
            "rk_efield": (C.c_int, [P, _F, _I, _I, _F, _F, _F, _F, _F, _F]),
            "rk_pcg": (C.c_int, [C.c_int, C.c_int, _I, _I, _F, _F, _F, _F, C.c_float, C.c_int, C.c_int, _I, _F]),
            "rk_xsec": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_float, _F, C.c_int, _F, _F, C.c_int]),
            "rk_kinematics": (C.c_int, [C.c_int, _F, _F, C.c_int]),
            "rk_mcc_ar": (C.c_int, [P, _F, _I, C.c_float, _F, _F, _F, _F, _F, _F, _F, _F, _LL, _I,
                                    _F, _F, _F, _F, _F, _F, _LL]),
            "rk_fluid_source": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _F, _F, _F, _F, _F, _F, _F]),
            "rk_oxy_collide": (C.c_int, [C.c_int, C.c_int, C.c_int, _I, C.c_float, _F, _F, _F, _F, C.c_int, _F,
                                         _F, _I, _F, _F, _F, C.c_int, _I, _F, _F, _LL]),
        }
        for k, (r, a) in sig.items():
            f = getattr(L, k)
            f.restype = r
            f.argtypes = a
        _lib = L
    return _lib


class RefError(RuntimeError):
    pass


def _check(rc):
    if rc != 0:
        raise RefError(f"reference harness error {rc}: {lib().rk_last_error().decode()}")


def _f(a):
    return a.ctypes.data_as(_F)


def _i(a):
    return a.ctypes.data_as(_I)


def f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def case_from_oracle(o, mpnc):
    """The rk_case of an oracle.Oracle (the same float constants it uses)."""
    c = o.c
    r = RkCase()
    r.ngx, r.ngy, r.nsp, r.mpnc = c.ngx, c.ngy, c.nsp, mpnc
    r.dt_dx, r.dt_dy = c.dt_dx, c.dt_dy
    for s in range(c.nsp):
        r.ascale[s], r.q_density[s], r.escale[s], r.np2c[s] = c.Ascale[s], c.q_density[s], c.Escale[s], c.np2c[s]
    return r


def cell_to_node(info):
    """node ID of every cell (cell = i * ncy + j -> i * ngy + j)."""
    cells = np.arange(info.Csize)
    i, j = cells // info.ncy, cells % info.ncy
    return (i * info.ngy + j).astype(np.int64)


class RefState:
    """Particles of all species in the reference layout."""

    def __init__(self, info, mpnc):
        self.info, self.mpnc = info, mpnc
        G, nsp = info.Gsize, info.nsp
        self.maxnp = mpnc * G
        n = nsp * self.maxnp
        self.pnc = np.zeros(nsp * G, np.int32)
        self.pnmc = np.zeros(nsp * G, np.int32)
        self.a = [np.zeros(n, np.float32) for _ in range(5)]
        self.cellid = np.zeros(n, np.int32)

    def index(self, s, node, k):
        return s * self.maxnp + node + k * self.info.Gsize


def to_ref(info, mpnc, species):
    """species: list over isp of (counts per cell, [x, y, vx, vy, vz]) in the
    oracle's cell order."""
    st = RefState(info, mpnc)
    node = cell_to_node(info)
    G = info.Gsize
    for s, (counts, arrs) in enumerate(species):
        counts = np.asarray(counts)
        assert counts.max(initial=0) <= mpnc, "more particles in a cell than slots"
        start = np.concatenate([[0], np.cumsum(counts)])
        # slot k of each particle inside its cell
        cell_of = np.repeat(np.arange(info.Csize), counts)
        k = np.arange(start[-1]) - start[cell_of]
        idx = s * st.maxnp + node[cell_of] + k * G
        for q in range(5):
            st.a[q][idx] = arrs[q]
        st.pnc[s * G + node] = counts
    return st


def from_ref(st, s, counts_at="pnc"):
    """(counts per cell, [x, y, vx, vy, vz]) of species s from the slots
    0 .. pnc-1 of every cell."""
    info = st.info
    G = info.Gsize
    node = cell_to_node(info)
    counts = st.pnc[s * G + node].astype(np.int32)
    start = np.concatenate([[0], np.cumsum(counts)])
    cell_of = np.repeat(np.arange(info.Csize), counts)
    k = np.arange(start[-1]) - start[cell_of]
    idx = s * st.maxnp + node[cell_of] + k * G
    return counts, [st.a[q][idx].copy() for q in range(5)]


def movers_from_ref(st, s):
    """(movers per cell, arrays, cell offsets) of species s: the r-th mover of
    a cell sits at slot mpnc - 1 - r (src/cuda_Move.cu:228)."""
    info = st.info
    G = info.Gsize
    node = cell_to_node(info)
    counts = st.pnmc[s * G + node].astype(np.int32)
    start = np.concatenate([[0], np.cumsum(counts)])
    cell_of = np.repeat(np.arange(info.Csize), counts)
    r = np.arange(start[-1]) - start[cell_of]
    idx = s * st.maxnp + node[cell_of] + (st.mpnc - 1 - r) * G
    return counts, [st.a[q][idx].copy() for q in range(5)], st.cellid[idx].copy()


# ------------------------------------------------------------------ entries
def move(rc, st, ex, ey):
    ex, ey = f32(ex), f32(ey)
    _check(lib().rk_move(C.byref(rc), _f(ex), _f(ey), _i(st.pnc), _i(st.pnmc), *[_f(a) for a in st.a],
                         _i(st.cellid)))


def set_timing(reps):
    """reps > 0: move() and deposit() also time their reference kernels
    over reps launches on restored inputs (the reference's launch shape)."""
    lib().rk_set_timing(int(reps))


def last_ms():
    """Mean kernel times (ms) of the last timed call: move() [MoveE_Basic];
    deposit() [DepositInitDensity, DepositAtom, DepositBoundary, SumSource]."""
    out = np.zeros(8, np.float32)
    lib().rk_last_ms(_f(out))
    return [float(v) for v in out]


def sortboundary(rc, st, sidx, cond_num):
    sidx = i32(sidx)
    cond = np.zeros(max(1, st.info.nsp * cond_num), np.float32)
    rearg = np.zeros(1, np.int32)
    _check(lib().rk_sortboundary(C.byref(rc), cond_num, _i(sidx), _i(st.pnc), _i(st.pnmc), *[_f(a) for a in st.a],
                                 _i(st.cellid), _f(cond), _i(rearg)))
    return cond[:st.info.nsp * cond_num], int(rearg[0])


def sort_probe(rc, st, sidx):
    out = np.zeros(8, np.int64)
    rl = np.zeros(2, np.int32)
    _check(lib().rk_sort_probe(C.byref(rc), _i(i32(sidx)), _i(st.pnc), _i(st.pnmc), _i(st.cellid),
                               out.ctypes.data_as(_LL), _i(rl)))
    return out, rl


def deposit(rc, st, face, boundary, cond_id, area, sigma_in=None, sigma_node_in=None):
    info = st.info
    G, nsp = info.Gsize, info.nsp
    den = np.zeros(nsp * G, np.float32)
    src = np.zeros(G, np.float32)
    sig = np.zeros(G, np.float32)
    si = None if sigma_in is None else f32(sigma_in)
    sn = None if sigma_node_in is None else f32(sigma_node_in)
    _check(lib().rk_deposit(C.byref(rc), _i(i32(face)), _i(i32(boundary)), _i(i32(cond_id)), _f(f32(area)),
                            _i(st.pnc), _f(st.a[0]), _f(st.a[1]), None if si is None else _f(si),
                            None if sn is None else _f(sn), _f(den), _f(src), _f(sig)))
    return den, src, sig


def efield(rc, geom, face, boundary, eps, den, sigma, phi):
    G = rc.ngx * rc.ngy
    sig = f32(sigma).copy()
    ex = np.zeros(G, np.float32)
    ey = np.zeros(G, np.float32)
    _check(lib().rk_efield(C.byref(rc), _f(f32(geom)), _i(i32(face)), _i(i32(boundary)), _f(f32(eps)),
                           _f(f32(den)), _f(sig), _f(f32(phi)), _f(ex), _f(ey)))
    return ex, ey, sig


def pcg(ai, aj, val, m, b, x0, tol2, nblocks=0, nthreads=512):
    """PCG_float; nblocks 0: the reference's own launch shape."""
    ai, aj, val, m, b = i32(ai), i32(aj), f32(val), f32(m), f32(b)
    x = f32(x0).copy()
    it = np.zeros(1, np.int32)
    ms = np.zeros(1, np.float32)
    n = b.size
    _check(lib().rk_pcg(n, aj.size, _i(ai), _i(aj), _f(val), _f(m), _f(b), _f(x), np.float32(tol2), nblocks, nthreads,
                        _i(it), _f(ms)))
    return x, int(it[0]), float(ms[0])


def xsec(gas, ch, n_logx, idlogx, table, width, engy):
    e = f32(engy)
    out = np.zeros(e.size, np.float32)
    _check(lib().rk_xsec(gas, ch, n_logx, np.float32(idlogx), _f(f32(table)), width, _f(e), _f(out), e.size))
    return out


def kinematics(kind, inp):
    inp = f32(inp)
    w = {0: 7, 1: 6, 2: 4}[kind]
    n = inp.size // w
    out = np.zeros(3 * n, np.float32)
    _check(lib().rk_kinematics(kind, _f(inp), _f(out), n))
    return out.reshape(n, 3)


def mcc_ar(rc, st, mcc, imcc, idlogx, vsave, table, sigv, collf, back_den1, back_vel1, fluid_n, u, start):
    info = st.info
    tnrct = imcc[3]
    mccr = np.zeros(info.Gsize * tnrct, np.float32)
    over = np.zeros(1, np.int64)
    startll = np.ascontiguousarray(start, np.int64)
    _check(lib().rk_mcc_ar(C.byref(rc), _f(f32(mcc)), _i(i32(imcc)), np.float32(idlogx), _f(f32(vsave)),
                           _f(f32(table)), _f(f32(sigv)), _f(f32(collf)), _f(f32(back_den1)), _f(f32(back_vel1)),
                           _f(f32(fluid_n)), _f(f32(u)), startll.ctypes.data_as(_LL), _i(st.pnc),
                           *[_f(a) for a in st.a], _f(mccr), over.ctypes.data_as(_LL)))
    return mccr.reshape(info.Gsize, tnrct), int(over[0])


def oxy_collide(gas, isp, imcc, idlogx, escale, vsave, table, sigv, collf, v, t, bv1, bv2, u):
    """One collision per collider through the reference's species handler."""
    nsp = 5 if gas == 2 else 4
    v = f32(v).reshape(-1, 3)
    n = v.shape[0]
    u = f32(u).reshape(n, -1)
    nu = u.shape[1]
    tnrct = imcc[2]
    cnt = np.zeros(n * nsp, np.int32)
    vout = np.zeros(n * nsp * 4 * 3, np.float32)
    mccr = np.zeros(n * tnrct, np.float32)
    over = np.zeros(1, np.int64)
    sg = f32(sigv)
    _check(lib().rk_oxy_collide(gas, isp, n, _i(i32(imcc)), np.float32(idlogx), _f(f32(escale)), _f(f32(vsave)),
                                _f(f32(table)), _f(sg), sg.size, _f(f32(collf)), _f(v), _i(i32(t)), _f(f32(bv1)),
                                _f(f32(bv2)), _f(u), nu, _i(cnt), _f(vout), _f(mccr), over.ctypes.data_as(_LL)))
    return cnt.reshape(n, nsp), vout.reshape(n, nsp, 4, 3), mccr.reshape(n, tnrct), int(over[0])


def fluid_source(gas, ngy, rates, rr, ave_e, fden, bd1, bd2):
    """The reference's Argon/Oxygen/ArO2_Update_Source on n nodes: rates
    [n, tnrct] averaged collision rates, ave_e [n] averaged electron density,
    fden [nfsp, n], bd1 and bd2 [n], rr [tnrct].  Returns (rates with the
    neutral channels filled, sources [nfsp, n])."""
    R = np.array(rates, np.float32, copy=True)
    n, tnrct = R.shape
    fden = np.ascontiguousarray(fden, np.float32)
    S = np.zeros(fden.shape, np.float32)
    _check(lib().rk_fluid_source(gas, n, ngy, tnrct, fden.shape[0], _f(R), _f(f32(rr)), _f(f32(ave_e)), _f(fden),
                                 _f(f32(bd1)), _f(f32(bd2)), _f(S)))
    return R, S
