"""ctypes binding of the CPU oracle (oracle/_build/liboracle.so).

Test infrastructure only: tests/, the smoke check and bench.py's CPU
baseline use this to compute the expected result of each step operator.
The oracle reads the case tables the library built (through hpic's table
export) and keeps its own particle and field state.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")

_F = C.POINTER(C.c_float)
_I = C.POINTER(C.c_int)
_D = C.POINTER(C.c_double)


class OrCase(C.Structure):
    _fields_ = [
        ("ngx", C.c_int), ("ngy", C.c_int), ("ncx", C.c_int), ("ncy", C.c_int), ("nsp", C.c_int),
        ("cond_numr", C.c_int), ("n_unknowns", C.c_int),
        ("dt_dx", C.c_float), ("dt_dy", C.c_float), ("dt", C.c_float), ("dx", C.c_float), ("dy", C.c_float),
        ("idx", C.c_float), ("idy", C.c_float), ("hdx", C.c_float), ("hdy", C.c_float), ("idxy", C.c_float),
        ("sidx", _I), ("boundary", _I), ("face", _I), ("cond_id", _I), ("eps", _F), ("dep_factor", _F),
        ("Ascale", C.c_float * 5), ("q_density", C.c_float * 5), ("Escale", C.c_float * 5),
        ("xsec", _F), ("n_logx", C.c_int), ("xw", C.c_int), ("idlogx", C.c_float),
        ("sigv", C.c_float * 32), ("th", C.c_float * 96), ("prob", _F), ("back_vel1", _F), ("vsave", _F),
        ("nvel", C.c_int), ("mcc_n", C.c_int), ("seed", C.c_uint64),
        ("st", _F), ("st_sym", _F), ("row_scale", _F), ("lap", _F),
        ("src_num", C.c_int), ("src_mid", C.c_int * 8), ("efield_flag", C.c_int * 8),
        ("src_dc", C.c_float * 8), ("src_ac", C.c_float * 8), ("src_2pif", C.c_float * 8),
        ("src_rphase", C.c_float * 8),
        ("pcg_tol2", C.c_float), ("pcg_max_iter", C.c_int), ("field_mode", C.c_int), ("pcg_rtol", C.c_double),
        ("pcg_cluster", C.c_int), ("pcg_block", C.c_int),
        ("fs_i0", C.c_int), ("fs_j0", C.c_int), ("fs_nx", C.c_int), ("fs_ny", C.c_int), ("fs_passes", C.c_int),
        ("fs_V", _F), ("fs_Vt", _F), ("fs_W", _F), ("fs_Wt", _F), ("fs_inv", _F),
        ("move_mode", C.c_int),
        ("gas", C.c_int), ("mcc_stride", C.c_int), ("mcc_all_species", C.c_int), ("eedf_every", C.c_int),
        ("dt_mcc", C.c_float),
        ("np2c", C.c_float * 5),
        ("back_den1", _F), ("back_den2", _F), ("back_vel2", _F),
        ("n_smt", C.c_int), ("dens_region", _I),
        ("n_diel", C.c_int), ("sig_mode", _I), ("area", _F),
        ("n_power", C.c_int), ("src_power", C.c_float * 8), ("cond_src_num", C.c_int * 8),
        ("cond_power_id", C.c_int * 8), ("pd_intv", C.c_int), ("pd_ratio", C.c_float),
        ("nfsp", C.c_int), ("fluid_on", C.c_int), ("n_ave", C.c_int), ("nxl", C.c_int), ("nyl", C.c_int),
        ("tnrct", C.c_int), ("dtc", C.c_float), ("denscale0", C.c_float),
        ("fluid_cell_den", _F), ("fluid_den", _F), ("xl", _I), ("yl", _I), ("xl_fg", _F), ("yl_fg", _F),
        ("gax", _F), ("gbx", _F), ("gay", _F), ("gby", _F), ("flux_x0", _F), ("flux_y0", _F), ("plasma", _I),
        ("rate_f", C.c_float * 96), ("rr", C.c_float * 96),
        ("external", C.c_int), ("cc_a", C.c_float * 20), ("lap_sig", C.c_float * 16), ("circuit_mode", C.c_int),
    ]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        P = C.c_void_p
        sig = {
            "or_sim_new": (P, [C.POINTER(OrCase), C.c_int]),
            "or_sim_free": (None, [P]),
            "or_set_particles": (None, [P, C.c_int, _I, _F, _F, _F, _F, _F]),
            "or_num_particles": (C.c_size_t, [P, C.c_int]),
            "or_get_particles": (None, [P, C.c_int, _I, _F, _F, _F, _F, _F]),
            "or_get_particles_d": (None, [P, C.c_int, _I, _D, _D, _D, _D, _D]),
            "or_num_movers": (C.c_size_t, [P, C.c_int]),
            "or_get_movers": (None, [P, C.c_int, _I, _F, _F, _F, _F, _F, C.POINTER(C.c_int8)]),
            "or_get_grid": (None, [P, C.c_int, P]),
            "or_set_grid": (None, [P, C.c_int, P]),
            "or_get_counters": (None, [P, _F, C.POINTER(C.c_uint), _I]),
            "or_walk_bound_hit": (C.c_int, [P]),
            "or_get_eedf": (None, [P, C.POINTER(C.c_uint64)]),
            "or_get_field_averages": (None, [P, P, P, P]),
            "or_math": (None, [C.c_int, _F, _F, _F, C.c_int]),
            "or_field": (None, [P, C.c_int64]),
            "or_move": (None, [P]),
            "or_sort": (None, [P]),
            "or_mcc": (None, [P, C.c_int64]),
            "or_deposit": (None, [P]),
            "or_deposit_basic": (None, [P]),
            "or_run": (None, [P, C.c_int64, C.c_int, C.c_int]),
            "or_get_averages": (None, [P, _D, _D, C.POINTER(C.c_int64)]),
            "or_set_script": (None, [P, C.c_int, _F, C.POINTER(C.c_int64), C.c_int]),
            "or_script_overrun": (C.c_longlong, [P]),
            "or_xsec": (None, [P, C.c_int, _F, _F, C.c_int]),
            "or_kinematics": (None, [P, C.c_int, _F, _F, C.c_int]),
            "or_collide_oxy": (C.c_int, [P, C.c_int, C.c_int, _F, C.c_float, C.c_float, _F, C.c_int, C.c_int, _I,
                                         _I, _F, _I, _F, _I]),
            "or_fluid_sweeps": (None, [P, C.c_int]),
            "or_fluid_sources": (None, [C.c_int, C.c_int, C.c_int, C.c_int, _F, _F, _F, _F, _F, _F, _F]),
            "or_num_threads": (C.c_int, []),
            "or_set_threads": (None, [C.c_int]),
        }
        for k, (r, a) in sig.items():
            f = getattr(L, k)
            f.restype = r
            f.argtypes = a
        _lib = L
    return _lib


def _fp(a):
    return a.ctypes.data_as(_F)


def _ip(a):
    return a.ctypes.data_as(_I)


class Oracle:
    """CPU restatement of one case.  `tables` is a callable name -> array
    (hpic.Case.table or hpic.Setup.table); `info` the case info."""

    GRID = dict(EX=0, EY=1, PHI=2, PHI_POIS=3, DEN=4, SOURCE=5, B=6, X=7, SURFACE_CHARGE=8, SIGMA=9, SOURCE_AC=10,
                FLUID_CELL_DEN=11, FLUID_DEN=12, FLUID_SOURCE=13, FLUID_FLUX_X=14, FLUID_FLUX_Y=15, CIRCUIT=16)

    def __init__(self, tables, info, opts, precision=32, pcg_cluster=1, pcg_block=512, field_mode=None,
                 fs_passes=None):
        self.info = info
        self.keep = {}
        t = tables
        sc = t("scalars")
        spc = t("species").reshape(-1, 16)
        src = t("sources")
        c = OrCase()
        c.ngx, c.ngy, c.ncx, c.ncy, c.nsp = info.ngx, info.ngy, info.ncx, info.ncy, info.nsp
        c.cond_numr, c.n_unknowns = info.cond_numr, info.n_unknowns
        dt, dx, dy = sc[0], sc[3], sc[4]
        c.dt = dt
        c.dt_dx = np.float32(dt) / np.float32(dx)
        c.dt_dy = np.float32(dt) / np.float32(dy)
        c.dx, c.dy, c.idx, c.idy, c.hdx, c.hdy, c.idxy = sc[3], sc[4], sc[5], sc[6], sc[7], sc[8], sc[9]

        def keep(name, arr, dtype):
            a = np.ascontiguousarray(arr, dtype=dtype)
            self.keep[name] = a
            return a.ctypes.data_as(_I if dtype == np.int32 else _F)

        c.sidx = keep("sidx", t("sidx"), np.int32)
        c.boundary = keep("boundary", t("boundary"), np.int32)
        c.face = keep("face", t("face"), np.int32)
        c.cond_id = keep("cond_id", t("cond_id"), np.int32)
        c.eps = keep("eps", (8.8542e-12 * t("eps_r").astype(np.float64)).astype(np.float32), np.float32)
        c.dep_factor = keep("dep", t("dep_factor"), np.float32)
        for s in range(info.nsp):
            c.Ascale[s] = spc[s, 7]
            c.q_density[s] = spc[s, 3]
            c.Escale[s] = spc[s, 6]
        c.xsec = keep("xsec", t("xsec"), np.float32)
        c.n_logx = int(sc[14])
        c.xw = self.keep["xsec"].size // c.n_logx
        c.idlogx = sc[15]
        sigv = t("sigv")
        for k in range(min(32, sigv.size)):
            c.sigv[k] = sigv[k]
        collf = t("collf").reshape(-1, 4)
        for k in range(min(96, collf.shape[0])):
            c.th[k] = collf[k, 2]
        c.gas = info.main_gas
        c.mcc_stride = info.mcc_stride
        c.mcc_all_species = 1 if opts.o2_all_species else 0
        c.eedf_every = max(0, opts.eedf_every)
        c.dt_mcc = sc[1]
        for s in range(info.nsp):
            c.np2c[s] = spc[s, 0]
        c.back_den1 = keep("bd1", t("back_den1"), np.float32)
        if info.main_gas != 0:
            c.back_den2 = keep("bd2", t("back_den2"), np.float32)
            c.back_vel2 = keep("bv2", t("back_vel2"), np.float32)
        # fluid species: the continuity solve and its sources
        fs = t("fluid_scalars")
        c.dtc, c.n_ave, c.nfsp, c.nxl, c.nyl = fs[0], int(fs[1]), int(fs[3]), int(fs[4]), int(fs[5])
        c.fluid_on = 0 if getattr(opts, "fluid_fixed", 0) else 1
        c.tnrct = info.n_reactions
        c.denscale0 = spc[0, 8]
        c.fluid_cell_den = keep("fcd", t("fluid_cell_den"), np.float32)
        c.fluid_den = keep("fd", t("fluid_den"), np.float32)
        c.xl = keep("xl", t("fluid_xlines"), np.int32)
        c.yl = keep("yl", t("fluid_ylines"), np.int32)
        c.xl_fg = keep("xlfg", t("fluid_xl_fg"), np.float32)
        c.yl_fg = keep("ylfg", t("fluid_yl_fg"), np.float32)
        for k in ("gax", "gbx", "gay", "gby", "flux_x0", "flux_y0"):
            setattr(c, k, keep(k, t("fluid_" + k), np.float32))
        c.plasma = keep("plasma", t("plasma_region"), np.int32)
        rf = t("fluid_rate_f")
        for k in range(min(96, rf.size)):
            c.rate_f[k] = rf[k]
            c.rr[k] = collf[k, 3]
        c.n_smt = info.n_smt
        c.dens_region = keep("dr", t("dens_region"), np.int32)
        c.n_diel = info.n_dielectric
        c.sig_mode = keep("sgm", t("sig_mode"), np.int32)
        c.area = keep("area", t("area"), np.float32)
        c.external = getattr(info, "circuit", 0)
        c.circuit_mode = getattr(opts, "circuit_mode", 0)
        if c.external:  # CC_a per conductor, then the Laplace bases' conductor charges
            tc = t("circuit")
            nc = info.cond_numr
            for i in range(nc):
                for q in range(5):
                    c.cc_a[i * 5 + q] = tc[i * 5 + q]
                for j in range(nc):
                    c.lap_sig[j * 4 + i] = tc[5 * nc + j * nc + i]
        c.n_power = info.power_driven
        pw = t("power")
        c.pd_intv, c.pd_ratio = int(pw[0]), pw[1]
        nsrc = info.n_sources
        for k in range(nsrc):
            c.src_power[k] = pw[2 + k]
        for k in range(info.cond_numr):
            c.cond_src_num[k] = int(pw[2 + nsrc + 2 * k])
            c.cond_power_id[k] = int(pw[3 + nsrc + 2 * k])
        c.prob = keep("prob", t("prob"), np.float32)
        c.back_vel1 = keep("bv1", t("back_vel1"), np.float32)
        c.vsave = keep("vsave", t("vsave"), np.float32)
        c.nvel = int(sc[12])
        c.mcc_n = int(sc[11])
        c.seed = opts.seed
        G = info.Gsize
        st_u = t("stencil").reshape(-1, 5)
        unk = t("unk_node")
        st = np.zeros((5, G), np.float32)
        sym = np.zeros((5, G), np.float32)
        scale = np.ones(G, np.float32)
        ii, jj = unk // info.ngy, unk % info.ngy
        d = (np.where((ii == 0) | (ii == info.ncx), 2, 1) * np.where((jj == 0) | (jj == info.ncy), 2, 1)).astype(
            np.float32)
        for k in range(5):
            st[k, unk] = st_u[:, k]
            sym[k, unk] = st_u[:, k] / d
        scale[unk] = np.float32(1.0) / d
        c.st = keep("st", st.ravel(), np.float32)
        c.st_sym = keep("st_sym", sym.ravel(), np.float32)
        c.row_scale = keep("scale", scale, np.float32)
        c.lap = keep("lap", t("lap"), np.float32)
        nsrc = (src.size - info.cond_numr) // 5
        c.src_num = nsrc
        for k in range(nsrc):
            c.src_mid[k] = int(src[5 * k])
            c.src_dc[k], c.src_ac[k], c.src_2pif[k], c.src_rphase[k] = src[5 * k + 1:5 * k + 5]
        for k in range(info.cond_numr):
            c.efield_flag[k] = int(src[5 * nsrc + k])
        c.pcg_tol2 = np.float32(sc[2]) * np.float32(sc[2])
        c.pcg_max_iter = opts.pcg_max_iter if opts.pcg_max_iter > 0 else 100000
        c.field_mode = opts.field_mode if field_mode is None else field_mode
        if c.field_mode == 2:
            fi = t("fs_info")
            if fi[0]:
                c.fs_i0, c.fs_j0, c.fs_nx, c.fs_ny = (int(v) for v in fi[1:5])
                if fs_passes is None:  # the library's default
                    rtol = opts.pcg_rtol if opts.pcg_rtol > 0 else 1e-8
                    fs_passes = opts.fs_passes if opts.fs_passes > 0 else (2 if rtol >= 1e-10 else 3)
                c.fs_passes = fs_passes
                c.fs_V = keep("fsV", t("fs_V"), np.float32)
                c.fs_Vt = keep("fsVt", t("fs_Vt"), np.float32)
                c.fs_W = keep("fsW", t("fs_W"), np.float32)
                c.fs_Wt = keep("fsWt", t("fs_Wt"), np.float32)
                c.fs_inv = keep("fsinv", t("fs_inv"), np.float32)
            else:
                c.field_mode = 1
        c.pcg_rtol = opts.pcg_rtol if opts.pcg_rtol > 0 else 1e-8
        c.move_mode = opts.move_mode
        c.pcg_cluster = pcg_cluster
        c.pcg_block = pcg_block
        self.c = c
        self.h = lib().or_sim_new(C.byref(c), precision)
        self.precision = precision

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_sim_free(self.h)
            self.h = None

    def set_particles(self, isp, counts, x, y, vx, vy, vz):
        arrs = [np.ascontiguousarray(a, np.float32) for a in (x, y, vx, vy, vz)]
        counts = np.ascontiguousarray(counts, np.int32)
        lib().or_set_particles(self.h, isp, _ip(counts), *[_fp(a) for a in arrs])

    def particles(self, isp):
        n = lib().or_num_particles(self.h, isp)
        counts = np.zeros(self.info.Csize, np.int32)
        arrs = [np.zeros(max(n, 1), np.float32) for _ in range(5)]
        lib().or_get_particles(self.h, isp, _ip(counts), *[_fp(a) for a in arrs])
        return counts, [a[:n] for a in arrs]

    def particles_d(self, isp):
        n = lib().or_num_particles(self.h, isp)
        counts = np.zeros(self.info.Csize, np.int32)
        arrs = [np.zeros(max(n, 1), np.float64) for _ in range(5)]
        lib().or_get_particles_d(self.h, isp, _ip(counts), *[a.ctypes.data_as(_D) for a in arrs])
        return counts, [a[:n] for a in arrs]

    def movers(self, isp):
        n = lib().or_num_movers(self.h, isp)
        counts = np.zeros(self.info.Csize, np.int32)
        arrs = [np.zeros(max(n, 1), np.float32) for _ in range(5)]
        codes = np.zeros(max(n, 1), np.int8)
        lib().or_get_movers(self.h, isp, _ip(counts), *[_fp(a) for a in arrs],
                            codes.ctypes.data_as(C.POINTER(C.c_int8)))
        return counts, [a[:n] for a in arrs], codes[:n]

    def grid(self, name):
        G, nsp = self.info.Gsize, self.info.nsp
        w = self.GRID[name]
        if w == 16:
            out = np.zeros(28, np.float32)
        elif w >= 11:
            nf, info = int(self.c.nfsp), self.info
            n = {11: nf * info.Csize, 12: nf * G, 13: nf * info.Csize, 14: nf * info.ngx * info.ncy, 15: nf * info.ncx * info.ngy}[w]
            out = np.zeros(n, np.float32)
        elif w <= 3:
            out = np.zeros(G, np.float32)
        elif w == 4:
            out = np.zeros(nsp * G, np.float64)
        elif w == 8:
            out = np.zeros(nsp * G, np.int64)
        elif w == 10:
            out = np.zeros(max(1, self.info.n_sources), np.float32)
        else:
            out = np.zeros(G, np.float64)
        lib().or_get_grid(self.h, w, out.ctypes.data_as(C.c_void_p))
        return out

    def set_grid(self, name, arr):
        w = self.GRID[name]
        dt = np.float32 if (w <= 3 or w >= 11) else np.int64 if w == 8 else np.float64
        a = np.ascontiguousarray(arr, dtype=dt)
        lib().or_set_grid(self.h, w, a.ctypes.data_as(C.c_void_p))

    def counters(self):
        cc = np.zeros(max(1, self.info.nsp * self.info.cond_numr), np.float32)
        mc = np.zeros(self.info.mcc_stride * self.info.Csize, np.uint32)
        it = np.zeros(2, np.int32)
        lib().or_get_counters(self.h, _fp(cc), mc.ctypes.data_as(C.POINTER(C.c_uint)), _ip(it))
        return cc, mc, it

    def walk_bound_hit(self):
        return bool(lib().or_walk_bound_hit(self.h))

    def far_max(self):
        return int(lib().or_far_max(self.h))

    def Field(self, tstep):
        lib().or_field(self.h, tstep)

    def Move(self):
        lib().or_move(self.h)

    def SortBoundary(self):
        lib().or_sort(self.h)

    def MCC(self, tstep):
        lib().or_mcc(self.h, tstep)

    def Deposit(self):
        """DEPOSIT: the per-step deposit, with the deck's smoothing passes."""
        lib().or_deposit(self.h)

    def DepositBasic(self):
        """Deposit_Basic: the initial deposit before the loop, no smoothing."""
        lib().or_deposit_basic(self.h)

    def run(self, tstep0, nsteps, accumulate=True):
        lib().or_run(self.h, tstep0, nsteps, 1 if accumulate else 0)

    def field_averages(self):
        """Running sums of the charge source, Ex and Ey (double[G] each)."""
        G = self.info.Gsize
        out = [np.zeros(G, np.float64) for _ in range(3)]
        lib().or_get_field_averages(self.h, *[a.ctypes.data_as(C.c_void_p) for a in out])
        return out

    def eedf(self):
        h = np.zeros(201, np.uint64)
        lib().or_get_eedf(self.h, h.ctypes.data_as(C.POINTER(C.c_uint64)))
        return h

    def set_script(self, u, start, by_species=False, pair_rl=0):
        """Scripted uniforms for the MCC (see oracle.h); u=None goes back to
        Philox.  pair_rl: mask of the kinematics calls (1 anewvel, 2 maxwellv,
        4 newvel_ionsc) whose two draws are taken right to left."""
        if u is None:
            lib().or_set_script(self.h, 0, None, None, 0)
            return
        self.keep["script_u"] = u = np.ascontiguousarray(u, np.float32)
        self.keep["script_s"] = st = np.ascontiguousarray(start, np.int64)
        flags = (1 if by_species else 0) | (int(pair_rl) << 1)
        lib().or_set_script(self.h, flags, _fp(u), st.ctypes.data_as(C.POINTER(C.c_int64)), st.size - 1)

    def script_overrun(self):
        return int(lib().or_script_overrun(self.h))

    def xsec(self, ch, engy):
        e = np.ascontiguousarray(engy, np.float32)
        out = np.zeros(e.size, np.float32)
        lib().or_xsec(self.h, ch, _fp(e), _fp(out), e.size)
        return out

    def kinematics(self, kind, inp):
        inp = np.ascontiguousarray(inp, np.float32)
        n = inp.size // {0: 7, 1: 6, 2: 4}[kind]
        out = np.zeros(3 * n, np.float32)
        lib().or_kinematics(self.h, kind, _fp(inp), _fp(out), n)
        return out.reshape(n, 3)

    def collide_oxy(self, isp, t, v, bv1, bv2, u, pair_rl=0):
        """One collision (Ar/O2 or O2 set) from the draws u: (channel, keep,
        velocity, born species[2], their velocities[2][3], O- removed)."""
        v = np.ascontiguousarray(v, np.float32)
        u = np.ascontiguousarray(u, np.float32)
        ch, keep, kill = C.c_int(0), C.c_int(0), C.c_int(0)
        vout = np.zeros(3, np.float32)
        bsp = np.zeros(2, np.int32)
        bv = np.zeros(6, np.float32)
        over = lib().or_collide_oxy(self.h, isp, t, _fp(v), np.float32(bv1), np.float32(bv2), _fp(u), u.size,
                                    int(pair_rl), C.byref(ch), C.byref(keep), _fp(vout), _ip(bsp), _fp(bv),
                                    C.byref(kill))
        return ch.value, bool(keep.value), vout, bsp, bv.reshape(2, 3), bool(kill.value), bool(over)

    def fluid_sweeps(self, nsteps):
        """The continuity solve alone, nsteps times, with the current sources."""
        lib().or_fluid_sweeps(self.h, nsteps)

    def averages(self):
        G, nsp = self.info.Gsize, self.info.nsp
        d = np.zeros(nsp * G, np.float64)
        p = np.zeros(G, np.float64)
        n = C.c_int64(0)
        lib().or_get_averages(self.h, d.ctypes.data_as(_D), p.ctypes.data_as(_D), C.byref(n))
        return d, p, n.value


def fluid_sources(gas, rates, fden, eden, bd1, bd2, rr):
    """The fluid sources of n nodes (include/hp_fluid.h): rates [n, tnrct],
    fden [nfsp, n], eden [n], bd1 and bd2 [n], rr [tnrct].  Returns (rates
    with the neutral channels filled, sources [nfsp, n])."""
    R = np.array(rates, np.float32, copy=True)
    n, tnrct = R.shape
    fden = np.ascontiguousarray(fden, np.float32)
    nfsp = fden.shape[0]
    S = np.zeros((nfsp, n), np.float32)
    f = [np.ascontiguousarray(a, np.float32) for a in (eden, bd1, bd2, rr)]
    lib().or_fluid_sources(gas, n, tnrct, nfsp, _fp(R), _fp(fden), *[_fp(a) for a in f], _fp(S))
    return R, S


def from_setup(setup, precision=32, field_mode=0, pcg_cluster=1, pcg_block=512):
    """Oracle for a hpic.Setup, loaded with its initial particles."""
    import hpic  # noqa: F401  (path set by the caller)
    opts = setup.opts
    opts.field_mode = field_mode
    o = Oracle(setup.table, setup.info, opts, precision, pcg_cluster, pcg_block)
    for s in range(setup.info.nsp):
        counts, arrs = setup.particles(s, layout=0)
        o.set_particles(s, counts, *arrs)
    return o
