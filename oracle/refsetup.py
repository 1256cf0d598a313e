"""A case for the oracle built without the product library (test and
baseline infrastructure only).

`oracle/_ref/ref_dump` runs the reference's own host set-up code on a deck:
InputRead, Geometry_setting, Source_setting, FieldSolverSetting and
GasSetting (src/start.c, src/load.c, src/Efield.c, src/PhysicsData.c,
src/Particle.c), the particle load included.  The few set-up steps the
reference runs in its CUDA host code are restated here from its sources:

* the null-collision maxima and electron sub-cycles of
  Set_NullCollisionTime_cuda (src/cuda_mcc.cu:202-276, the Ar set);
* the Laplace basis of each conductor, PCG_SOLVER_Laplace +
  PCG_Deposit_Lap (src/cuda_Field.cu:182-236,648-655): A x = cond_b[k],
  conductor k's nodes at 1 V;
* the gas temperature and background density, the TA x = temp_b solve,
  PCG_Deposit_Temp and Calculate_1GasPara (src/cuda_Field.cu:221-233,
  656-669);
* the deposit's boundary factors of DepositBoundary (src/cuda_Deposit.cu:
  277-288), the per-cell collision probabilities of Direct_Argon_*
  (src/cuda_mccAr.cu:54-56,189) and the cell-sorted particle order of
  Copy_HCPtoGCP (src/cuda_Particle.cu:28-58).

The solves are direct (SciPy) in FP64, where the reference iterates in FP32
to its tolerance.  `RefSetup` offers the interface the oracle reads
(`table`, `info`, `opts`, `particles`).  The Ar reaction set only.
"""
import os
import subprocess
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DUMP = os.path.join(HERE, "_ref", "ref_dump")

NPERTORR = 8.3221e20
DBL_MIN = 1e-200
# enum BoundaryCondition / BoundaryType (inc/def.h:21-38)
DIRICHLET, NEUMANN = 1, 2
F_LEFT, F_RIGHT, F_UP, F_DOWN, F_UL, F_UR, F_LL, F_LR, F_NONE = range(9)

GGA = np.dtype([("Boundary", "<i4"), ("CondID", "<i4"), ("Face", "<i4"), ("DensRegion", "<i4"), ("Area", "<f4"),
                ("Temp", "<f4"), ("BackDen1", "<f4"), ("BackVel1", "<f4"), ("BackDen2", "<f4"),
                ("BackVel2", "<f4"), ("Lap_Pot", "<f4"), ("Pois_Pot", "<f4"), ("Ex", "<f4"), ("Ey", "<f4")])
GCA = np.dtype([("PlasmaRegion", "<i4"), ("eps_r", "<f4"), ("eps", "<f4")])


def available():
    return os.path.exists(REF_DUMP)


def _meta(path):
    m = {}
    for line in open(path):
        k, v = line.split()
        try:
            m[k] = int(v)
        except ValueError:
            m[k] = float(v)
    return m


def _read(d, name, dtype):
    return np.fromfile(os.path.join(d, name + ".bin"), dtype=dtype)


def _solve(ai, aj, val, b):
    import scipy.sparse as sps
    import scipy.sparse.linalg as spl
    n = ai.size - 1
    A = sps.csr_matrix((val.astype(np.float64), aj - 1, ai - 1), shape=(n, n)).tocsc()
    return spl.spsolve(A, np.asarray(b, np.float64).T).T


class RefSetup:
    """The case of one deck, as the oracle reads it."""

    def __init__(self, deck_text, seed, field_mode=0, move_mode=1, pcg_rtol=1e-8):
        if not available():
            raise RuntimeError("oracle/_ref/ref_dump is not built (make -C oracle ref)")
        with tempfile.TemporaryDirectory() as d:
            deck = os.path.join(d, "deck.json")
            with open(deck, "w") as f:
                f.write(deck_text)
            out = os.path.join(d, "out")
            os.mkdir(out)
            subprocess.run([REF_DUMP, deck, str(int(seed)), out], check=True, stdout=subprocess.DEVNULL,
                           stderr=subprocess.DEVNULL)
            self._deck, self._seed = deck, int(seed)
            self._load(out, seed, field_mode, move_mode, pcg_rtol)

    def _fluid(self, d, temp, m, t):
        """The fluid species' set-up: the reference's Fluid_Setting, diffusion
        and Gummel coefficients and initial fluxes (src/Fluid.c:3-224,
        src/cuda_Fluid.cu:3-95,185-298), which need the gas temperature of every
        node, so ref_dump runs again with it."""
        fd = d + "_fluid"
        os.mkdir(fd)
        tp = os.path.join(fd, "temps.bin")
        temp.astype(np.float32).tofile(tp)
        subprocess.run([REF_DUMP, self._deck, str(self._seed), fd, tp], check=True, stdout=subprocess.DEVNULL,
                       stderr=subprocess.DEVNULL)
        ngx, ngy, ncx, ncy, nfsp = m["ngx"], m["ngy"], m["ncx"], m["ncy"], m["nfsp"]
        G, C = ngx * ngy, ncx * ncy
        cell = _read(fd, "fl_den0", np.float32)
        # Sync_Fluid_GFCtoGFG_forDen (src/cuda_Fluid.cu:321-339): node (i, j) of
        # cell (i, j), and node (i+1, j+1) of the last row and column; nodes
        # (0, ncy) and (ncx, 0) are written by nothing in the reference (its
        # memory there is never set) and are 0 here
        node = np.zeros((max(nfsp, 1), ngx, ngy), np.float32)
        cg = cell.reshape(max(nfsp, 1), ncx, ncy) if nfsp else np.zeros((1, ncx, ncy), np.float32)
        node[:, :ncx, :ncy] = cg
        node[:, ncx, 1:] = cg[:, ncx - 1, :]
        node[:, 1:, ncy] = cg[:, :, ncy - 1]
        t["fluid_cell_den"] = cell
        t["fluid_den"] = node.reshape(-1)[:max(nfsp, 1) * G] if nfsp else np.zeros(G, np.float32)
        xl, yl = _read(fd, "fl_xlines", np.int32), _read(fd, "fl_ylines", np.int32)
        t["fluid_xlines"], t["fluid_ylines"] = xl, yl
        for k in ("xl_fg", "yl_fg", "D", "gax", "gbx", "gay", "gby", "flux_x0", "flux_y0"):
            t["fluid_" + k] = _read(fd, "fl_" + k, np.float32)
        dt = np.float32(m["dt"])
        t["fluid_scalars"] = np.array([dt * np.float32(m["DT_CONTI"]), m["N_ave"], m["DT_CONTI"], nfsp, xl.size // 3,
                                       yl.size // 3], np.float32)
        # Argon_Update_Source's rate factors (src/cuda_Diagnostic.cu:634-642):
        # the electron channels 0-6 and 8 at Denscale / N_ave / dt
        rf = np.zeros(m["TnRct"], np.float32)
        f0 = np.float32(np.float32(m["sp0_Denscale"]) / np.float32(m["N_ave"])) / dt
        rf[0:7] = f0
        rf[8] = f0
        t["fluid_rate_f"] = rf

    # ------------------------------------------------------------ assembly
    def _load(self, d, seed, field_mode, move_mode, pcg_rtol):
        m = _meta(os.path.join(d, "meta.txt"))
        if m["MainGas"] != 0:
            raise NotImplementedError("the Ar reaction set only")
        ngx, ngy, ncx, ncy = m["ngx"], m["ngy"], m["ncx"], m["ncy"]
        G, C, nsp = ngx * ngy, ncx * ncy, m["nsp"]
        gga = _read(d, "gga", GGA)
        gca = _read(d, "gca", GCA)
        t = {}
        t["sidx"] = _read(d, "sidx", np.int32)
        aidx = t["a_idx"] = _read(d, "aidx", np.int32)
        for k, name in (("Boundary", "boundary"), ("Face", "face"), ("CondID", "cond_id"),
                        ("DensRegion", "dens_region")):
            t[name] = np.ascontiguousarray(gga[k])
        t["area"] = np.ascontiguousarray(gga["Area"])
        t["eps_r"] = np.ascontiguousarray(gca["eps_r"])
        ai, aj, val = _read(d, "ai", np.int32), _read(d, "aj", np.int32), _read(d, "a_val", np.float32)
        t["ai"], t["aj"], t["a_val"] = ai, aj, val
        t["matm"] = _read(d, "matm", np.float32)
        N = m["A_size"]
        cond_numr = m["CondNUMR"]
        cond_b = _read(d, "cond_b", np.float32).reshape(cond_numr, N)
        temp_b, ta_val = _read(d, "temp_b", np.float32), _read(d, "ta_val", np.float32)
        xsec = t["xsec"] = _read(d, "xsec", np.float32)
        collf = t["collf"] = _read(d, "collf", np.float32)
        t["vsave"] = _read(d, "vsave", np.float32)
        n_logx = m["N_LOGX"]
        W = xsec.size // n_logx
        # node stencil (W, S, C, N, E) of every unknown: its CSR row
        unk = np.nonzero(aidx)[0].astype(np.int32)
        unk = unk[np.argsort(aidx[unk])]
        st = np.zeros((N, 5), np.float32)
        rows = np.repeat(np.arange(N), np.diff(ai))
        off = unk[aj - 1].astype(np.int64) - unk[rows]
        slot = np.full(off.size, -1)
        for k, o_ in enumerate((-ngy, -1, 0, 1, ngy)):
            slot[off == o_] = k
        if (slot < 0).any():
            raise ValueError("the reference matrix is not a 5-point stencil")
        st[rows, slot] = val
        t["stencil"], t["unk_node"] = st.ravel(), unk
        # Laplace bases and gas temperature (direct solves of the reference's systems)
        xs = _solve(ai, aj, val, cond_b)
        xs = xs.reshape(cond_numr, N) if cond_numr > 1 else xs.reshape(1, N)
        lap = np.zeros((cond_numr, G), np.float32)
        has = aidx > 0
        for k in range(cond_numr):
            lap[k, has] = xs[k, aidx[has] - 1].astype(np.float32)
            lap[k, (~has) & (gga["CondID"] == k + 1)] = 1.0
        t["lap"] = lap.ravel()
        temp = gga["Temp"].copy()
        xt = _solve(ai, aj, ta_val, temp_b)
        temp[has] = xt[aidx[has] - 1].astype(np.float32)
        t["node_temp"] = temp
        pres, mass = m["bg0_Pres"], m["bg0_mass"]
        dr = gga["DensRegion"] != 0
        T = temp.astype(np.float64)
        bd1 = np.zeros(G, np.float32)
        bv1 = np.zeros(G, np.float32)
        bd1[dr] = (NPERTORR * np.float64(np.float32(pres)) / (T[dr] * 8.6142e-5 + DBL_MIN)).astype(np.float32)
        bv1[dr] = np.sqrt(T[dr] * 1.38e-23 / np.float64(np.float32(mass))).astype(np.float32)
        t["back_den1"], t["back_vel1"] = bd1, bv1
        t["back_den2"] = np.zeros(G, np.float32)
        t["back_vel2"] = np.zeros(G, np.float32)
        nfsp = m["nfsp"]
        t["plasma_region"] = np.ascontiguousarray(gca["PlasmaRegion"])
        self._fluid(d, temp, m, t)
        fl = t["fluid_den"].reshape(max(nfsp, 1), G)
        # DepositBoundary's factors
        face, bnd, cid = gga["Face"], gga["Boundary"], gga["CondID"]
        dep = np.ones(G, np.float32)
        dep[np.isin(face, [F_LEFT, F_RIGHT, F_UP, F_DOWN])] *= 2
        dep[np.isin(face, [F_UL, F_UR, F_LL, F_LR])] *= 4
        dep[bnd == NEUMANN] *= 2
        dep[(bnd == DIRICHLET) & (face != F_NONE) & (cid != 0)] *= 2
        t["dep_factor"] = dep
        t["sig_mode"] = np.zeros(G, np.int32)
        # Set_NullCollisionTime_cuda, Ar: sigma-v maxima over the table, electron sub-cycles
        tab = xsec.reshape(n_logx, W).astype(np.float32)
        m_e, m_i = np.float32(m["sp0_mass"]), np.float32(m["sp1_mass"])
        sig = [tab[:, 2] + tab[:, 3] + tab[:, 4] + tab[:, 5], tab[:, 6], tab[:, 7] + tab[:, 8]]
        sigv = np.zeros(3, np.float32)
        for k, mass_k in ((0, m_e), (1, m_e), (2, m_i)):
            best = np.float32(0)
            for r in range(n_logx):
                v = np.sqrt(2 * 1.602e-19 * np.float64(tab[r, 1]) / np.float64(mass_k)) * np.float64(sig[k][r])
                best = np.float32(max(np.float64(best), v))
            sigv[k] = best
        dt = np.float32(m["dt"])
        bg0 = np.float32(m["bg0_InitDens"])
        fg0 = np.float32(m["fg0_InitDens"]) if nfsp else np.float32(0)
        # 1.0 - exp(-1 * dt * sigma_v * n): the product in float, exp in double
        T0 = np.float32(1.0 - np.exp(np.float64(np.float32(-1) * dt * sigv[0] * bg0)))
        T1 = np.float32(1.0 - np.exp(np.float64(np.float32(-1) * dt * sigv[1] * fg0)))
        col0 = np.float32(T0 + T1)
        if col0 > np.float32(0.08):
            mcc_n = int(np.ceil(np.float64(col0 / np.float32(0.08))))
            dt_mcc = np.float32(dt * np.float32(1 / np.float32(mcc_n)))
        else:
            mcc_n, dt_mcc = 1, dt
        t["sigv"] = sigv
        cells = np.arange(C)
        cnode = (cells // ncy) * ngy + cells % ncy
        def expf(x):  # a correctly rounded float exp
            return np.exp(x.astype(np.float64)).astype(np.float32)

        P1 = np.float32(1) - expf(np.float32(-1) * dt_mcc * sigv[0] * bd1[cnode])
        P2 = P1 + np.float32(1) - expf(np.float32(-1) * dt_mcc * sigv[1] * fl[0][cnode])
        Pi = np.float32(1) - expf(np.float32(-1) * dt * sigv[2] * bd1[cnode])
        t["prob"] = np.concatenate([P1, P2, Pi]).astype(np.float32)
        # scalars and species, in the layout the oracle reads
        t["scalars"] = np.array([dt, dt_mcc, m["PCGtol"], m["dx"], m["dy"], m["idx"], m["idy"], m["hdx"], m["hdy"],
                                 m["idxy"], m["zlength"], mcc_n, m["h_nvel"], m["TnRct"], n_logx, m["idLOGX"]],
                                np.float32)
        spc = np.zeros((nsp, 16), np.float32)
        for s in range(nsp):
            spc[s] = [m[f"sp{s}_np2c"], m[f"sp{s}_mass"], m[f"sp{s}_q"], m[f"sp{s}_q_density"], m[f"sp{s}_vti"],
                      m[f"sp{s}_qm"], m[f"sp{s}_Escale"], m[f"sp{s}_Ascale"], m[f"sp{s}_Denscale"],
                      m[f"sp{s}_MCCscale"], m[f"sp{s}_MAXNP"], m[f"sp{s}_Temp"], m[f"sp{s}_InitDens"],
                      m[f"sp{s}_np"], 0, 0]
        t["species"] = spc.ravel()
        src = []
        nsrc = m["SrcNUM"]
        for k in range(nsrc):
            src += [m[f"src{k}_MID"], m[f"src{k}_DC"], m[f"src{k}_AC"],
                    np.float32(2 * np.pi) * np.float32(m[f"src{k}_FREQ"]), m[f"src{k}_RPHASE"]]
        src += [m[f"efield_flag{k}"] for k in range(cond_numr)]
        t["sources"] = np.array(src, np.float32)
        t["power"] = np.zeros(2 + nsrc + 2 * cond_numr, np.float32)
        self.t = t
        self.info = types.SimpleNamespace(ngx=ngx, ngy=ngy, ncx=ncx, ncy=ncy, Gsize=G, Csize=C, nsp=nsp, main_gas=0,
                                          cond_numr=cond_numr, n_unknowns=N, mcc_stride=8, n_smt=0, n_dielectric=0,
                                          n_sources=nsrc, power_driven=0, n_reactions=m["TnRct"],
                                          mcc_subcycles=mcc_n, dt=float(dt), dx=m["dx"], dy=m["dy"])
        self.opts = types.SimpleNamespace(seed=int(seed), field_mode=field_mode, pcg_rtol=pcg_rtol, pcg_max_iter=0,
                                          o2_all_species=0, move_mode=move_mode, fs_passes=0, eedf_every=0,
                                          gas_temp_mode=0)
        # Copy_HCPtoGCP: cells from the integer part of the position, a stable
        # order inside each cell (a frand() of exactly 1 stays in the last cell)
        self.p = []
        for s in range(nsp):
            x = _read(d, f"p{s}_x", np.float32)
            y = _read(d, f"p{s}_y", np.float32)
            xi = x.astype(np.int32)
            yi = y.astype(np.int32)
            ox = x - xi.astype(np.float32)
            oy = y - yi.astype(np.float32)
            over_x, over_y = xi >= ncx, yi >= ncy
            xi[over_x], ox[over_x] = ncx - 1, np.float32(0.99999994)
            yi[over_y], oy[over_y] = ncy - 1, np.float32(0.99999994)
            cell = xi * ncy + yi
            order = np.argsort(cell, kind="stable")
            counts = np.bincount(cell, minlength=C).astype(np.int32)
            arrs = [ox[order], oy[order]] + [_read(d, f"p{s}_{c}", np.float32)[order] for c in ("vx", "vy", "vz")]
            self.p.append((counts, arrs))

    # ------------------------------------------------------------ interface
    def table(self, name, dtype=None):
        a = self.t[name]
        return a if dtype is None else a.astype(dtype)

    def particles(self, isp, layout=0):
        if layout != 0:
            raise ValueError("cell-sorted layout only")
        return self.p[isp]
