"""Python binding of libhpic (the C ABI declared in include/hpic.h).

This mirrors the reference's host interface for the step: a case is built
from a JSON deck in the reference's format, and the per-step operators keep
the reference's names (Field = PCG_SOLVER + EFIELD, Move, SortBoundary, MCC,
Deposit; inc/main.h:25-32).  Every call goes through ctypes into the
compiled library; there is no Python or CPU implementation of any operator
here, and a missing library raises instead of falling back.
"""
import ctypes as C
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG, "lib", "libhpic.so")
DECK_DIR = os.path.join(PKG, "decks")

HP_OK, HP_ERR_ARG, HP_ERR_DECK, HP_ERR_CUDA, HP_ERR_OOM, HP_ERR_UNSUPPORTED, HP_ERR_DEVICE, HP_ERR_CAPACITY, \
    HP_ERR_NO_CUDA = range(9)
STATUS_CELL_OVERFLOW, STATUS_NONFINITE, STATUS_PCG_NOCONV, STATUS_WAIT_TIMEOUT = 1, 2, 4, 8
STATUS_WALK_BOUND, STATUS_SURFACE_OVERFLOW = 0x10, 0x20

# conductors an external circuit may have (HP_CIRCUIT_MAX, include/hp_circuit.h)
CIRCUIT_MAX = 4
GRID = dict(EX=0, EY=1, PHI=2, PHI_POIS=3, DEN=4, SOURCE=5, PCG_X=6, PCG_B=7, AVE_DEN=8, AVE_PHI=9,
            COND_CHARGE=10, MCC_COUNT=11, EEDF=12, AVE_SOURCE=13, AVE_EX=14, AVE_EY=15,
            SURFACE_CHARGE=16, SIGMA=17, SOURCE_AC=18, POWER_STATE=19, FLUID_CELL_DEN=20, FLUID_DEN=21,
            FLUID_SOURCE=22, FLUID_FLUX_X=23, FLUID_FLUX_Y=24, FLUID_STATE=25, CIRCUIT=26)
SIGMA_FRAC_BITS = 28  # fixed-point fraction bits of SURFACE_CHARGE (particle weights)
POWER_STATE_BYTES = 8 * 8 * 3 + 4 * 8 * 2 + 8  # PowerState: surf, old, old2 (double[8]); power, count; flags
EEDF_BINS, EEDF_DE = 200, 0.25  # electron energy histogram: 0.25 eV bins from 0, one overflow bin
TABLE = dict(sidx=0, a_idx=1, boundary=2, face=3, cond_id=4, area=5, back_den1=6, back_vel1=7, lap=8,
             stencil=9, vsave=10, xsec=11, collf=12, sigv=13, dens_region=14, prob=15, eps_r=16,
             back_den2=17, back_vel2=18, a_val=19, ai=20, aj=21, matm=22, cond_b=23, temp_b=24, ta_val=25,
             species=26, node_temp=27, dep_factor=28, fluid_den=29, scalars=30, sources=31, unk_node=32,
             fs_info=33, fs_V=34, fs_Vt=35, fs_W=36, fs_Wt=37, fs_inv=38, sig_mode=39, power=40,
             fluid_cell_den=41, fluid_xlines=42, fluid_ylines=43, fluid_xl_fg=44, fluid_yl_fg=45, fluid_gax=46,
             fluid_gbx=47, fluid_gay=48, fluid_gby=49, fluid_flux_x0=50, fluid_flux_y0=51, fluid_D=52,
             fluid_scalars=53, fluid_rate_f=54, plasma_region=55, circuit=56)
TABLE_DTYPE = {0: np.int32, 1: np.int32, 2: np.int32, 3: np.int32, 4: np.int32, 14: np.int32, 20: np.int32,
               21: np.int32, 32: np.int32, 33: np.int32, 39: np.int32, 42: np.int32, 43: np.int32, 55: np.int32}


class HpicError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"hpic status {status}: {msg}")
        self.status = status


class CaseOpts(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("cap_per_cell", C.c_int), ("field_mode", C.c_int),
                ("pcg_rtol", C.c_double), ("pcg_max_iter", C.c_int), ("o2_all_species", C.c_int),
                ("device", C.c_int), ("gas_temp_mode", C.c_int), ("move_mode", C.c_int),
                ("fs_passes", C.c_int), ("eedf_every", C.c_int), ("gpu_load", C.c_int), ("fluid_fixed", C.c_int),
                ("circuit_mode", C.c_int)]


class CaseInfo(C.Structure):
    _fields_ = [("ngx", C.c_int), ("ngy", C.c_int), ("ncx", C.c_int), ("ncy", C.c_int), ("Gsize", C.c_int),
                ("Csize", C.c_int), ("nsp", C.c_int), ("main_gas", C.c_int), ("cond_numr", C.c_int),
                ("n_unknowns", C.c_int), ("cap", C.c_int * 8), ("mcc_subcycles", C.c_int), ("dt", C.c_double),
                ("dx", C.c_double), ("dy", C.c_double), ("tstep", C.c_int64), ("device_bytes", C.c_size_t),
                ("pcg_cluster", C.c_int), ("pcg_block", C.c_int), ("field_mode", C.c_int), ("mcc_stride", C.c_int),
                ("n_smt", C.c_int), ("n_dielectric", C.c_int), ("n_sources", C.c_int),
                ("power_driven", C.c_int), ("n_reactions", C.c_int), ("n_fluid", C.c_int), ("circuit", C.c_int)]


class Tune(C.Structure):
    _fields_ = [("warps_per_block_particles", C.c_int), ("pcg_block", C.c_int), ("pcg_cluster_max", C.c_int),
                ("move_unroll", C.c_int), ("mcc_cells_per_warp", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class KernelStat(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("launches", C.c_int), ("ms", C.c_double)]


class Gcp(C.Structure):  # the reference's GCP record (inc/def.h)
    _fields_ = [("CellID", C.c_int), ("x", C.c_float), ("y", C.c_float), ("vx", C.c_float), ("vy", C.c_float),
                ("vz", C.c_float)]


class Gpg(C.Structure):  # the reference's GPG record
    _fields_ = [("PtNumInCell", C.c_int), ("PtNumMoveInterCell", C.c_int), ("MaxPtNumInCell", C.c_int),
                ("PtNumMCCInCell", C.c_int), ("PtNullMCCInCell", C.c_int), ("den", C.c_float),
                ("smt_den", C.c_float), ("sum_den", C.c_float), ("ave_den", C.c_float), ("sigma", C.c_float)]


class Gga(C.Structure):  # the reference's GGA record
    _fields_ = [("Boundary", C.c_int), ("CondID", C.c_int), ("Face", C.c_int), ("DensRegion", C.c_int)] + \
        [(k, C.c_float) for k in ("Area", "Temp", "BackDen1", "BackVel1", "BackDen2", "BackVel2", "Lap_Pot",
                                   "Pois_Pot", "Ex", "Ey")]


GCP_DTYPE = np.dtype([("CellID", "i4"), ("x", "f4"), ("y", "f4"), ("vx", "f4"), ("vy", "f4"), ("vz", "f4")])
GPG_DTYPE = np.dtype([("PtNumInCell", "i4"), ("PtNumMoveInterCell", "i4"), ("MaxPtNumInCell", "i4"),
                      ("PtNumMCCInCell", "i4"), ("PtNullMCCInCell", "i4"), ("den", "f4"), ("smt_den", "f4"),
                      ("sum_den", "f4"), ("ave_den", "f4"), ("sigma", "f4")])
GGA_DTYPE = np.dtype([("Boundary", "i4"), ("CondID", "i4"), ("Face", "i4"), ("DensRegion", "i4")] +
                     [(k, "f4") for k in ("Area", "Temp", "BackDen1", "BackVel1", "BackDen2", "BackVel2", "Lap_Pot",
                                          "Pois_Pot", "Ex", "Ey")])


class ServerOpts(C.Structure):
    _fields_ = [("mem_budget_bytes", C.c_size_t), ("max_slots", C.c_int), ("steps_per_launch", C.c_int),
                ("case_opts", CaseOpts)]


class Result(C.Structure):
    _fields_ = [("request_id", C.c_int64), ("error", C.c_int), ("status", C.c_uint32), ("steps", C.c_int64),
                ("particle_pushes", C.c_int64), ("t_submit", C.c_double), ("t_admit", C.c_double),
                ("t_done", C.c_double), ("ngx", C.c_int), ("ngy", C.c_int), ("nsp", C.c_int)]


_lib = None

_P = C.c_void_p
_F = C.POINTER(C.c_float)
_I = C.POINTER(C.c_int)

_SIGS = {
    "hp_last_error": (C.c_char_p, []),
    "hp_case_opts_default": (None, [C.POINTER(CaseOpts)]),
    "hp_setup_build": (C.c_int, [C.c_char_p, C.c_size_t, C.POINTER(CaseOpts), C.POINTER(_P)]),
    "hp_setup_destroy": (None, [_P]),
    "hp_setup_get_info": (C.c_int, [_P, C.POINTER(CaseInfo)]),
    "hp_setup_get_table": (C.c_int, [_P, C.c_int, _P, C.c_size_t, C.POINTER(C.c_size_t)]),
    "hp_setup_get_particles": (C.c_int, [_P, C.c_int, C.c_int, _I, _F, _F, _F, _F, _F, C.c_size_t,
                                         C.POINTER(C.c_size_t)]),
    "hp_case_create": (C.c_int, [C.c_char_p, C.c_size_t, C.POINTER(CaseOpts), C.POINTER(_P)]),
    "hp_case_create_from_setup": (C.c_int, [_P, C.POINTER(CaseOpts), C.POINTER(_P)]),
    "hp_case_destroy": (C.c_int, [_P]),
    "hp_case_get_info": (C.c_int, [_P, C.POINTER(CaseInfo)]),
    "hp_case_status": (C.c_int, [_P, C.POINTER(C.c_uint32)]),
    "hp_case_set_tstep": (C.c_int, [_P, C.c_int64]),
    "hp_Field": (C.c_int, [_P, _P]),
    "hp_Move": (C.c_int, [_P, _P]),
    "hp_SortBoundary": (C.c_int, [_P, _P]),
    "hp_MCC": (C.c_int, [_P, _P]),
    "hp_Deposit": (C.c_int, [_P, _P]),
    "hp_step": (C.c_int, [_P, C.c_int, _P]),
    "hp_step_kernels": (C.c_int, [_P, C.POINTER(C.c_int)]),
    "hp_case_set_tune": (C.c_int, [_P, _P]),
    "hp_case_get_tune": (C.c_int, [_P, _P]),
    "hp_batch_step_kernels": (C.c_int, [_P, C.POINTER(C.c_int)]),
    "hp_profile_step": (C.c_int, [_P, C.c_int, _P, C.POINTER(KernelStat), C.c_int, C.POINTER(C.c_int)]),
    "hp_export_gcp": (C.c_int, [_P, C.c_int, C.c_int, _P, _P]),
    "hp_import_gcp": (C.c_int, [_P, C.c_int, C.c_int, _P, _P]),
    "hp_export_gga": (C.c_int, [_P, _P]),
    "hp_Deposit_noalloc": (C.c_int, [_P, _P, _P]),
    "hp_get_particles": (C.c_int, [_P, C.c_int, _I, _F, _F, _F, _F, _F, C.c_size_t, C.POINTER(C.c_size_t)]),
    "hp_set_particles": (C.c_int, [_P, C.c_int, _I, _F, _F, _F, _F, _F]),
    "hp_get_movers": (C.c_int, [_P, C.c_int, _I, _F, _F, _F, _F, _F, C.POINTER(C.c_int8), C.c_size_t,
                                C.POINTER(C.c_size_t)]),
    "hp_get_grid": (C.c_int, [_P, C.c_int, _P, C.c_size_t]),
    "hp_set_grid": (C.c_int, [_P, C.c_int, _P, C.c_size_t]),
    "hp_reset_averages": (C.c_int, [_P]),
    "hp_get_mcc_rates": (C.c_int, [_P, C.POINTER(C.c_float), C.c_size_t]),
    "hp_get_average_count": (C.c_int, [_P, C.POINTER(C.c_int64)]),
    "hp_last_pcg_iters": (C.c_int, [_P, _I, _I]),
    "hp_last_field_residual": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "hp_case_pushes": (C.c_int, [_P, C.POINTER(C.c_int64)]),
    "hp_case_slot_changes": (C.c_int, [_P, C.POINTER(C.c_int64)]),
    "hp_case_save": (C.c_int, [_P, C.c_char_p]),
    "hp_case_load": (C.c_int, [_P, C.c_char_p]),
    "hp_get_table": (C.c_int, [_P, C.c_int, _P, C.c_size_t, C.POINTER(C.c_size_t)]),
    "hp_batch_create": (C.c_int, [C.POINTER(_P), C.c_int, C.POINTER(_P)]),
    "hp_batch_destroy": (C.c_int, [_P]),
    "hp_batch_step": (C.c_int, [_P, C.c_int, _P]),
    "hp_batch_set_tune": (C.c_int, [_P, C.POINTER(Tune)]),
    "hp_batch_get_tune": (C.c_int, [_P, C.POINTER(Tune)]),
    "hp_batch_autotune": (C.c_int, [_P, _P]),
    "hp_server_opts_default": (None, [C.POINTER(ServerOpts)]),
    "hp_server_create": (C.c_int, [C.POINTER(ServerOpts), C.POINTER(_P)]),
    "hp_server_destroy": (C.c_int, [_P]),
    "hp_server_submit": (C.c_int, [_P, C.c_char_p, C.c_size_t, C.c_int64, C.c_uint64, C.POINTER(C.c_int64)]),
    "hp_server_poll": (C.c_int, [_P, _P, _I]),
    "hp_server_take_result": (C.c_int, [_P, C.POINTER(Result), C.POINTER(C.c_double), C.c_size_t,
                                        C.POINTER(C.c_double), C.c_size_t, _I]),
}


def lib():
    """Load libhpic.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is missing: build it with `make -C hybrid-final_b200`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(st):
    if st != HP_OK:
        raise HpicError(st, lib().hp_last_error().decode(errors="replace"))


def default_opts(**kw):
    o = CaseOpts()
    lib().hp_case_opts_default(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def _fptr(a):
    return a.ctypes.data_as(_F)


def _iptr(a):
    return a.ctypes.data_as(_I)


def deck_text(deck):
    """A deck given as a dict, a JSON string or a path to a .json file."""
    import json
    if isinstance(deck, dict):
        return json.dumps(deck)
    if isinstance(deck, str) and deck.lstrip().startswith("{"):
        return deck
    with open(deck) as f:
        return f.read()


class Setup:
    """Host-side case tables built from a deck (no GPU needed)."""

    def __init__(self, deck, **opts):
        self.opts = default_opts(**opts)
        text = deck_text(deck).encode()
        h = _P()
        _check(lib().hp_setup_build(text, len(text), C.byref(self.opts), C.byref(h)))
        self.h = h
        info = CaseInfo()
        _check(lib().hp_setup_get_info(self.h, C.byref(info)))
        self.info = info

    def __del__(self):
        if getattr(self, "h", None):
            lib().hp_setup_destroy(self.h)
            self.h = None

    def table(self, name, dtype=None):
        what = TABLE[name] if isinstance(name, str) else name
        need = C.c_size_t(0)
        _check(lib().hp_setup_get_table(self.h, what, None, 0, C.byref(need)))
        dt = dtype or TABLE_DTYPE.get(what, np.float32)
        out = np.zeros(need.value // np.dtype(dt).itemsize, dtype=dt)
        _check(lib().hp_setup_get_table(self.h, what, out.ctypes.data_as(_P), need.value, C.byref(need)))
        return out

    def particles(self, isp, layout=0):
        n = C.c_size_t(0)
        info = self.info
        np_ = int(self.table("species").reshape(-1, 16)[isp, 13])
        cells = np.zeros(info.Csize if layout == 0 else max(np_, 1), dtype=np.int32)
        arrs = [np.zeros(max(np_, 1), dtype=np.float32) for _ in range(5)]
        _check(lib().hp_setup_get_particles(self.h, isp, layout, _iptr(cells), *[_fptr(a) for a in arrs],
                                            max(np_, 1), C.byref(n)))
        k = n.value
        return (cells if layout == 0 else cells[:k]), [a[:k] for a in arrs]


class Case:
    """One discharge case resident on the GPU."""

    def __init__(self, deck=None, setup=None, **opts):
        self.opts = default_opts(**opts)
        h = _P()
        if setup is not None:
            _check(lib().hp_case_create_from_setup(setup.h, C.byref(self.opts), C.byref(h)))
        else:
            text = deck_text(deck).encode()
            _check(lib().hp_case_create(text, len(text), C.byref(self.opts), C.byref(h)))
        self.h = h
        info = CaseInfo()
        _check(lib().hp_case_get_info(self.h, C.byref(info)))
        self.info = info

    def close(self):
        if getattr(self, "h", None):
            lib().hp_case_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown: the library may be gone already
            pass

    # per-step operators (reference names)
    def Field(self, stream=None):
        _check(lib().hp_Field(self.h, stream))

    def Move(self, stream=None):
        _check(lib().hp_Move(self.h, stream))

    def SortBoundary(self, stream=None):
        _check(lib().hp_SortBoundary(self.h, stream))

    def MCC(self, stream=None):
        _check(lib().hp_MCC(self.h, stream))

    def Deposit(self, stream=None):
        _check(lib().hp_Deposit(self.h, stream))

    def step(self, n=1, stream=None):
        _check(lib().hp_step(self.h, n, stream))

    def set_tstep(self, t):
        _check(lib().hp_case_set_tstep(self.h, t))

    def tstep(self):
        info = CaseInfo()
        _check(lib().hp_case_get_info(self.h, C.byref(info)))
        return info.tstep

    def status(self):
        s = C.c_uint32(0)
        _check(lib().hp_case_status(self.h, C.byref(s)))
        return s.value

    def pcg_iters(self):
        a, b = C.c_int(0), C.c_int(0)
        _check(lib().hp_last_pcg_iters(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def field_residual(self):
        r = C.c_double(0)
        _check(lib().hp_last_field_residual(self.h, C.byref(r)))
        return r.value

    def tune(self):
        t = Tune()
        _check(lib().hp_case_get_tune(self.h, C.byref(t)))
        return t.as_dict()

    def set_tune(self, **kw):
        cur = self.tune()
        cur.update(kw)
        t = Tune(**cur)
        _check(lib().hp_case_set_tune(self.h, C.byref(t)))

    def step_kernels(self):
        """Kernels one step launches (after the first step captured it)."""
        n = C.c_int(0)
        _check(lib().hp_step_kernels(self.h, C.byref(n)))
        return n.value

    def pushes(self):
        n = C.c_int64(0)
        _check(lib().hp_case_pushes(self.h, C.byref(n)))
        return n.value

    def save(self, path):
        """Checkpoint: the reference's V000 dump plus the exact-resume extension."""
        _check(lib().hp_case_save(self.h, str(path).encode()))

    def load(self, path):
        """Resume from a checkpoint written by save() for the same deck and options."""
        _check(lib().hp_case_load(self.h, str(path).encode()))

    def slot_changes(self):
        """Pushed particles whose slot changed (cumulative)."""
        n = C.c_int64(0)
        _check(lib().hp_case_slot_changes(self.h, C.byref(n)))
        return n.value

    def particles(self, isp):
        n = C.c_size_t(0)
        counts = np.zeros(self.info.Csize, dtype=np.int32)
        _check(lib().hp_get_particles(self.h, isp, _iptr(counts), None, None, None, None, None, 0, C.byref(n)))
        k = max(n.value, 1)
        arrs = [np.zeros(k, dtype=np.float32) for _ in range(5)]
        _check(lib().hp_get_particles(self.h, isp, _iptr(counts), *[_fptr(a) for a in arrs], k, C.byref(n)))
        return counts, [a[:n.value] for a in arrs]

    def movers(self, isp):
        n = C.c_size_t(0)
        counts = np.zeros(self.info.Csize, dtype=np.int32)
        _check(lib().hp_get_movers(self.h, isp, _iptr(counts), None, None, None, None, None, None, 0, C.byref(n)))
        k = max(n.value, 1)
        arrs = [np.zeros(k, dtype=np.float32) for _ in range(5)]
        codes = np.zeros(k, dtype=np.int8)
        _check(lib().hp_get_movers(self.h, isp, _iptr(counts), *[_fptr(a) for a in arrs],
                                   codes.ctypes.data_as(C.POINTER(C.c_int8)), k, C.byref(n)))
        return counts, [a[:n.value] for a in arrs], codes[:n.value]

    def set_particles(self, isp, counts, x, y, vx, vy, vz):
        arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (x, y, vx, vy, vz)]
        counts = np.ascontiguousarray(counts, dtype=np.int32)
        _check(lib().hp_set_particles(self.h, isp, _iptr(counts), *[_fptr(a) for a in arrs]))

    def grid(self, name):
        info = self.info
        G, nsp, nf = info.Gsize, info.nsp, info.n_fluid
        sizes = dict(EX=(G, np.float32), EY=(G, np.float32), PHI=(G, np.float32), PHI_POIS=(G, np.float32),
                     DEN=(nsp * G, np.float64), SOURCE=(G, np.float64),
                     PCG_X=(G, np.float32 if self.opts.field_mode == 0 else np.float64),
                     PCG_B=(G, np.float64), AVE_DEN=(nsp * G, np.float64), AVE_PHI=(G, np.float64),
                     COND_CHARGE=(nsp * info.cond_numr, np.float32), MCC_COUNT=(info.mcc_stride * info.Csize, np.uint32),
                     EEDF=(EEDF_BINS + 1, np.uint64), AVE_SOURCE=(G, np.float64), AVE_EX=(G, np.float64),
                     AVE_EY=(G, np.float64),
                     SURFACE_CHARGE=(nsp * G if info.n_dielectric else 0, np.int64),
                     SIGMA=(G if (info.n_dielectric or info.power_driven) else 0, np.float64),
                     SOURCE_AC=(info.n_sources, np.float32),
                     POWER_STATE=(POWER_STATE_BYTES if info.power_driven else 0, np.uint8),
                     FLUID_CELL_DEN=(nf * info.Csize, np.float32), FLUID_DEN=(nf * G, np.float32),
                     FLUID_SOURCE=(nf * info.Csize, np.float32), FLUID_FLUX_X=(nf * info.ngx * info.ncy, np.float32),
                     FLUID_FLUX_Y=(nf * info.ncx * info.ngy, np.float32),
                     FLUID_STATE=(G * 8 + info.Csize * info.mcc_stride * 4 + 3 * info.Csize * 4, np.uint8),
                     CIRCUIT=(7 * CIRCUIT_MAX if info.circuit else 0, np.float32))
        n, dt = sizes[name]
        out = np.zeros(n, dtype=dt)
        _check(lib().hp_get_grid(self.h, GRID[name], out.ctypes.data_as(_P), out.nbytes))
        return out

    def set_grid(self, name, arr):
        arr = np.ascontiguousarray(arr)
        _check(lib().hp_set_grid(self.h, GRID[name], arr.ctypes.data_as(_P), arr.nbytes))

    def reset_averages(self):
        _check(lib().hp_reset_averages(self.h))

    def mcc_rates(self):
        """Averaged collision rates [Gsize, TnRct] (the reference's ave_MCC_rate)."""
        info = self.info
        out = np.zeros(info.Gsize * info.n_reactions, np.float32)
        _check(lib().hp_get_mcc_rates(self.h, out.ctypes.data_as(C.POINTER(C.c_float)), out.size))
        return out.reshape(info.Gsize, info.n_reactions)

    def average_count(self):
        n = C.c_int64(0)
        _check(lib().hp_get_average_count(self.h, C.byref(n)))
        return n.value

    def table(self, name, dtype=None):
        what = TABLE[name] if isinstance(name, str) else name
        need = C.c_size_t(0)
        _check(lib().hp_get_table(self.h, what, None, 0, C.byref(need)))
        dt = dtype or TABLE_DTYPE.get(what, np.float32)
        out = np.zeros(need.value // np.dtype(dt).itemsize, dtype=dt)
        _check(lib().hp_get_table(self.h, what, out.ctypes.data_as(_P), need.value, C.byref(need)))
        return out

    def n_particles(self):
        return [int(self.particles_count(s)) for s in range(self.info.nsp)]

    def movers_count(self, isp):
        """Movers parked in the cells by the last Move (their number only)."""
        n = C.c_size_t(0)
        _check(lib().hp_get_movers(self.h, isp, None, None, None, None, None, None, None, 0, C.byref(n)))
        return n.value

    def export_gcp(self, isp, mpnc):
        """Species isp in the reference's layout: (GCP records [mpnc*Gsize],
        GPG records [Gsize]) as numpy structured arrays."""
        G = self.info.Gsize
        gcp = np.zeros(mpnc * G, GCP_DTYPE)
        gpg = np.zeros(G, GPG_DTYPE)
        _check(lib().hp_export_gcp(self.h, isp, mpnc, gcp.ctypes.data_as(_P), gpg.ctypes.data_as(_P)))
        return gcp, gpg

    def import_gcp(self, isp, mpnc, gcp, gpg):
        gcp = np.ascontiguousarray(gcp, GCP_DTYPE)
        gpg = np.ascontiguousarray(gpg, GPG_DTYPE)
        _check(lib().hp_import_gcp(self.h, isp, mpnc, gcp.ctypes.data_as(_P), gpg.ctypes.data_as(_P)))

    def export_gga(self):
        gga = np.zeros(self.info.Gsize, GGA_DTYPE)
        _check(lib().hp_export_gga(self.h, gga.ctypes.data_as(_P)))
        return gga

    def profile(self, n=1, stream=None):
        """Per-kernel device times of n op-by-op steps (hp_profile_step):
        [(name, launches, ms)] in the order the kernels first ran."""
        cap = 64
        out = (KernelStat * cap)()
        k = C.c_int(0)
        _check(lib().hp_profile_step(self.h, int(n), stream, out, cap, C.byref(k)))
        return [(out[i].name.decode(), out[i].launches, out[i].ms) for i in range(min(k.value, cap))]

    def particles_count(self, isp):
        n = C.c_size_t(0)
        counts = np.zeros(self.info.Csize, dtype=np.int32)
        _check(lib().hp_get_particles(self.h, isp, _iptr(counts), None, None, None, None, None, 0, C.byref(n)))
        return n.value


class Batch:
    """Independent cases advanced with one launch per phase."""

    def __init__(self, cases):
        self.cases = list(cases)
        arr = (_P * len(self.cases))(*[c.h for c in self.cases])
        h = _P()
        _check(lib().hp_batch_create(arr, len(self.cases), C.byref(h)))
        self.h = h

    def step(self, n=1, stream=None):
        _check(lib().hp_batch_step(self.h, n, stream))

    def step_kernels(self):
        n = C.c_int(0)
        _check(lib().hp_batch_step_kernels(self.h, C.byref(n)))
        return n.value

    def tune(self):
        t = Tune()
        _check(lib().hp_batch_get_tune(self.h, C.byref(t)))
        return t.as_dict()

    def set_tune(self, **kw):
        cur = self.tune()
        cur.update(kw)
        t = Tune(**cur)
        _check(lib().hp_batch_set_tune(self.h, C.byref(t)))

    def autotune(self, stream=None):
        _check(lib().hp_batch_autotune(self.h, stream))

    def close(self):
        if getattr(self, "h", None):
            lib().hp_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown: the library may be gone already
            pass


class Server:
    """The served form: a request loop over resident cases (continuous
    batching).  `submit` queues a deck; `poll` runs one scheduling round
    (admission by device footprint and free slots, a few batched steps,
    retirement); `results` pops finished requests with their time-averaged
    densities and potential."""

    def __init__(self, mem_budget_bytes=None, max_slots=None, steps_per_launch=None, **case_opts):
        o = ServerOpts()
        lib().hp_server_opts_default(C.byref(o))
        if mem_budget_bytes is not None:
            o.mem_budget_bytes = int(mem_budget_bytes)
        if max_slots is not None:
            o.max_slots = int(max_slots)
        if steps_per_launch is not None:
            o.steps_per_launch = int(steps_per_launch)
        for k, v in case_opts.items():
            setattr(o.case_opts, k, v)
        self.opts = o
        h = _P()
        _check(lib().hp_server_create(C.byref(o), C.byref(h)))
        self.h = h
        self.shapes = {}

    def submit(self, deck, nsteps, seed=1):
        text = deck_text(deck)
        raw = text.encode()
        rid = C.c_int64(0)
        _check(lib().hp_server_submit(self.h, raw, len(raw), int(nsteps), int(seed), C.byref(rid)))
        d = json.loads(text)
        g = d["Geometry"]["SystemSpec"]
        self.shapes[rid.value] = (int(g["NumGridx"]), int(g["NumGridy"]))
        return rid.value

    def poll(self, stream=None):
        n = C.c_int(0)
        _check(lib().hp_server_poll(self.h, stream, C.byref(n)))
        return n.value

    def results(self):
        """Finished requests: list of (Result, ave_den[nsp, G], ave_phi[G])."""
        out = []
        while True:
            r = Result()
            got = C.c_int(0)
            # buffers sized for the largest case submitted to this server
            cap_g = max((a * b for a, b in self.shapes.values()), default=1)
            den = np.zeros(5 * cap_g)
            phi = np.zeros(cap_g)
            _check(lib().hp_server_take_result(self.h, C.byref(r), den.ctypes.data_as(C.POINTER(C.c_double)),
                                               den.size, phi.ctypes.data_as(C.POINTER(C.c_double)), phi.size,
                                               C.byref(got)))
            if not got.value:
                return out
            G = r.ngx * r.ngy
            out.append((r, den[: r.nsp * G].reshape(r.nsp, G).copy() if r.nsp else den[:0],
                        phi[:G].copy()))

    def run(self, stream=None, max_rounds=10 ** 9):
        """Poll until every submitted request has finished; returns results."""
        res = []
        for _ in range(max_rounds):
            pending = self.poll(stream)
            res += self.results()
            if pending == 0:
                break
        return res + self.results()

    def close(self):
        if getattr(self, "h", None):
            lib().hp_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown: the library may be gone already
            pass
