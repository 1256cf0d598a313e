"""Benchmark: particle-pushes/s of the PIC/MCC step on B200.

One step = Field (Poisson solve + E), Move, SortBoundary, MCC, Deposit for
every particle of the case; one particle-push = one particle advanced through
one step.  Default workload (N=1): the single large Ar case of the precision
form, 513x257 nodes (16 cm x 8 cm), 200 macro-particles per cell per species
(about 26M electrons + 26M Ar+), 100 V at 13.56 MHz, 50 mTorr, FP32
particles, FP64 charge grid and FP64-refined field solve (field_mode 2).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank advances its own replica of the case (one case does
not shard: replicas only); value = pushes of all ranks / max rank time.
`--impl reference` times the reference's CPU path on this host's cores, on the
same workload: the reference's own set-up code (oracle/_ref) and the CPU
restatement of its step (the reference has no CPU step of its own), with its
own numerics; it loads nothing of this library.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "hybrid-final_b200")
sys.path.insert(0, PKG)

METRIC = "particle-pushes/s batched vs plain at ≤1% FP64 error; p50/p99 case latency"
UNIT = "particle-pushes/s"
# the workload decks' averaging window: AverageIter = steps per RF period
AVERAGE_ITER = 400
# Move: read and write x, y, vx, vy (32 B) for every particle, plus vz (8 B)
# for each particle whose slot changes (a push leaves vz as it is)
MOVE_BYTES_PER_PARTICLE = 32
MOVE_BYTES_PER_SLOT_CHANGE = 8

WORKLOADS = {
    "ar_513x257_200ppc": dict(ngx=513, ngy=257, xlen=0.16, ylen=0.08, ppc=200, voltage=100.0, pressure=0.05),
    "ar_257x129_200ppc": dict(ngx=257, ngy=129, xlen=0.08, ylen=0.04, ppc=200, voltage=100.0, pressure=0.05),
    "ar_129x65_50ppc": dict(ngx=129, ngy=65, xlen=0.04, ylen=0.02, ppc=50, voltage=100.0, pressure=0.05),
    # the Ar/O2 case's gas, pressure, voltage and densities on the 129x65 grid (FP64 check)
    "aro2_129x65_50ppc": dict(ngx=129, ngy=65, xlen=0.04, ylen=0.02, ppc=50, voltage=200.0, pressure=0.1,
                              gas="ArO2", te=3.0, ions={"Ar+": 1e15, "O2+": 2e14, "O+": 0.0, "O-": 2e14}),
    # 80/20 Ar/O2 at 100 mTorr, 200 V: e 3 eV, Ar+ 1e15, O2+ 2e14, O+ 0, O- 2e14 m^-3
    "aro2_257x129_100ppc": dict(ngx=257, ngy=129, xlen=0.08, ylen=0.04, ppc=100, voltage=200.0, pressure=0.1,
                                gas="ArO2", te=3.0, ions={"Ar+": 1e15, "O2+": 2e14, "O+": 0.0, "O-": 2e14}),
}


def _decks():
    """hpic/decks.py loaded on its own (plain Python deck writer), so that the
    reference arm imports nothing of the library."""
    import importlib.util
    path = os.path.join(REPO, "hybrid-final_b200", "hpic", "decks.py")
    spec = importlib.util.spec_from_file_location("case_decks", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def make_deck(w):
    ccp_deck = _decks().ccp_deck
    extra = {}
    if w.get("gas", "Ar") != "Ar":
        extra = dict(gas=w["gas"], te_ev=w["te"], ion_density=w["ions"], aro2_ratio=(80, 20))
    return ccp_deck(w["ngx"], w["ngy"], w["xlen"], w["ylen"], ppc=w["ppc"], voltage=w["voltage"],
                    pressure_torr=w["pressure"], **extra)


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for k, n in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(n)
        med = float(np.median(sm)) if sm else None
        return {"sm_mhz": med, "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def dist_init(n_gpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as td
        torch.cuda.set_device(local)
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        dist = td
    return rank, world, local, dist


def allreduce(dist, v, op, device="cuda"):
    if dist is None:
        return v
    import torch
    t = torch.tensor([float(v)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def replica_throughput(dist, units, ms, device="cuda"):
    """Whole-job throughput of independent replicas: the units every rank
    processed over the slowest rank's device time.  Returns (units/s, max ms,
    total units)."""
    ms_max = allreduce(dist, ms, "max", device)
    units_all = allreduce(dist, units, "sum", device)
    return units_all / (ms_max * 1e-3), ms_max, units_all


def move_traffic(workload):
    """dram bytes per k_move launch from the committed ncu summary, if any."""
    return kernel_traffic("k_move", workload)


def kernel_traffic(kernel, workload):
    """dram bytes per launch of a kernel (read + write) from the committed ncu
    summary of the workload (profiles/dram_per_kernel_<workload>.md), if any."""
    path = os.path.join(REPO, "profiles", f"dram_per_kernel_{workload}.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith(f"dram_bytes_per_launch {kernel}:"):
            return float(line.split(":")[1].split()[0])
    return None


def kernel_rooflines(case, stream, peak, peak_kind, workload, steps=3):
    """Per-kernel device times of op-by-op steps (hp_profile_step: CUDA events
    around every launch on the launching stream) and the HBM rooflines of
    the kernels with an algorithmic byte count:
      k_move           32 B per particle + 8 B per slot change
      k_sort_push      41 B per mover (5 floats read and written, the code read)
      k_deposit_cells  8 B per particle (x, y) + 32 B per (species, cell) corner sums
      k_pcg(_grid)     40 B per unknown per inner iteration (x, r, p, Ap, the
                       stencil diagonal), field modes 0 and 1
    Returns (kernels, rooflines)."""
    info = case.info
    nsp = info.nsp
    parts = sum(case.particles_count(s) for s in range(nsp))
    ch0 = case.slot_changes()
    stats = case.profile(steps, stream)
    changes = (case.slot_changes() - ch0) / steps
    movers = sum(case.movers_count(s) for s in range(nsp))  # those of the last step
    total = sum(ms for _, _, ms in stats)
    kernels = [dict(name=n, launches_per_step=l / steps, ms_per_step=ms / steps, share=ms / total)
               for n, l, ms in sorted(stats, key=lambda t: -t[2])]
    bytes_per_launch = {
        "k_move": 32.0 * parts + 8.0 * changes,
        "k_sort_push": 41.0 * movers,
        "k_deposit_cells": 8.0 * parts + 32.0 * nsp * info.Csize,
    }
    inner, outer = case.pcg_iters()
    if inner > 0:  # the cluster solve (k_pcg) or the whole-GPU cooperative one (k_pcg_grid)
        bytes_per_launch["k_pcg"] = bytes_per_launch["k_pcg_grid"] = 40.0 * info.n_unknowns * inner
    rooflines = []
    for n, l, ms in stats:
        if n not in bytes_per_launch or l == 0:
            continue
        t = ms / l * 1e-3
        ach = bytes_per_launch[n] / t / 1e9
        r = dict(kernel=n, bound="hbm", achieved=ach, peak=peak, unit="GB/s", frac=ach / peak, peak_source=peak_kind,
                 algorithmic_bytes_per_launch=bytes_per_launch[n], us_per_launch=t * 1e6,
                 traffic=kernel_traffic(n, workload))
        if n.startswith("k_pcg"):
            r.update(inner_iterations=inner, outer_passes=outer, us_per_iteration=t * 1e6 / max(inner, 1),
                     unknowns=info.n_unknowns)
        rooflines.append(r)
    return kernels, rooflines


def peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d["hbm_gbs"], "measured"
    return 6650.0, "fallback"


def cpu_baseline(setup, case_opts, budget_s=20.0, what="CPU restatement"):
    """The CPU restatement (oracle, FP32 form) on this host: a bounded number
    of full steps of the same case."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle
    o = oracle.Oracle(setup.table, setup.info, case_opts, 32, field_mode=case_opts.field_mode)
    for s in range(setup.info.nsp):
        counts, arrs = setup.particles(s, layout=0)
        o.set_particles(s, counts, *arrs)
    o.DepositBasic()
    pushes, t_used, steps = 0, 0.0, 0
    while steps < 1 or (t_used < budget_s and steps < 20):
        n = sum(int(oracle.lib().or_num_particles(o.h, s)) for s in range(setup.info.nsp))
        t0 = time.perf_counter()
        o.run(steps, 1, accumulate=False)
        t_used += time.perf_counter() - t0
        pushes += n
        steps += 1
        if t_used > budget_s:
            break
    return dict(value=pushes / t_used, unit=UNIT, cores=int(oracle.lib().or_num_threads()), kind="port",
                sample=f"{steps} full step(s) of the same case ({pushes} particle-pushes) on the host, "
                       f"{what} in FP32, {t_used:.1f} s")


SPECIES = {"Ar": ["e", "Ar+"], "ArO2": ["e", "Ar+", "O2+", "O+", "O-"]}


def fp64_check(stream, workload="ar_129x65_50ppc", steps=800):
    """Error of the precision form against the FP64 oracle over two RF
    periods, on the reference's CPU-sized Ar case (129x65 nodes, 4 cm x 2 cm,
    50 particles per cell and species, 100 V, 50 mTorr) or the 80/20 Ar/O2
    case on the same grid (100 mTorr, 200 V): relative L2 error of the
    time-averaged density of every species (n_i: all positive ions), of the
    potential, and of the electron energy distribution (sampled every 4th
    step) as total-variation distance and relative error of the mean energy.
    The GPU runs the bench's numerics (FP32 particles, FP64 charge grid,
    field_mode 2); the oracle runs the same case and draws in FP64 on the
    host."""
    import hpic
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle
    w = WORKLOADS[workload]
    opts = dict(field_mode=2, gas_temp_mode=1, move_mode=1, eedf_every=4)
    S = hpic.Setup(make_deck(w), seed=77, **opts)
    c = hpic.Case(setup=S, seed=77, **opts)
    c.step(steps, stream)
    n = c.average_count()
    d32 = c.grid("AVE_DEN").reshape(c.info.nsp, -1) / n
    p32 = c.grid("AVE_PHI") / n
    h32 = c.grid("EEDF").astype(np.float64)
    status = c.status()
    c.close()
    # the sampling floor: the same precision form with another seed (other
    # particle draws), against the first run
    S2 = hpic.Setup(make_deck(w), seed=78, **opts)
    c2 = hpic.Case(setup=S2, seed=78, **opts)
    c2.step(steps, stream)
    n2 = c2.average_count()
    d32b = c2.grid("AVE_DEN").reshape(c2.info.nsp, -1) / n2
    p32b = c2.grid("AVE_PHI") / n2
    c2.close()
    del S2
    t0 = time.perf_counter()
    o = oracle.from_setup(S, 64, field_mode=2)
    o.c.move_mode = 1
    o.DepositBasic()
    o.run(0, steps, accumulate=True)
    d, p, m = o.averages()
    d64, p64 = d.reshape(S.info.nsp, -1) / m, p / m
    h64 = o.eedf().astype(np.float64)

    def rel(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))
    names = SPECIES[w.get("gas", "Ar")]
    pos = [k for k, nm in enumerate(names) if nm.endswith("+")]
    pe, qe = h32 / h32.sum(), h64 / h64.sum()
    ebin = (np.arange(pe.size) + 0.5) * hpic.EEDF_DE
    out = dict(case=workload, steps=steps, rf_periods=steps / 400, tolerance=0.01,
               rel_l2_ave_n_e=rel(d32[0], d64[0]), rel_l2_ave_n_i=rel(d32[pos].sum(0), d64[pos].sum(0)),
               rel_l2_ave_phi=rel(p32, p64))
    floor = dict(rel_l2_ave_n_e=rel(d32b[0], d32[0]), rel_l2_ave_n_i=rel(d32b[pos].sum(0), d32[pos].sum(0)),
                 rel_l2_ave_phi=rel(p32b, p32))
    if len(names) > 2:
        for k, nm in enumerate(names[1:], 1):
            if np.linalg.norm(d64[k]) > 0:
                out[f"rel_l2_ave_n_{nm}"] = rel(d32[k], d64[k])
                floor[f"rel_l2_ave_n_{nm}"] = rel(d32b[k], d32[k])
    # the difference between two FP32 runs that differ only in their seed:
    # an FP32-vs-FP64 error at or below it is sampling noise, not precision
    out["seed_to_seed"] = floor
    out.update(eedf_tv=round(0.5 * float(np.abs(pe - qe).sum()), 6),
               eedf_mean_energy_rel=round(abs(float(pe @ ebin) / float(qe @ ebin) - 1.0), 6),
               device_status=int(status), fp64_oracle_s=round(time.perf_counter() - t0, 1))
    return out


def run_ours(args, rank, world, local, dist):
    import torch

    import hpic
    torch.cuda.set_device(local)
    w = WORKLOADS[args.workload]
    deck = make_deck(w)
    seed = 1000 + rank
    setup = hpic.Setup(deck, seed=seed, field_mode=args.field_mode, gas_temp_mode=1, move_mode=args.move_mode)
    case = hpic.Case(setup=setup, seed=seed, field_mode=args.field_mode, move_mode=args.move_mode, device=local)
    stream = torch.cuda.current_stream().cuda_stream
    # warm-up (graph capture happens on the first call)
    case.step(args.warmup, stream)
    # the fluid species' continuity solve starts after the first averaging
    # window (one RF period, AverageIter steps; the reference's rule): step
    # through it untimed so that every timed step is a steady-state step
    spin_up = max(0, AVERAGE_ITER + 2 - args.warmup) if case.info.n_fluid > 0 else 0
    case.step(spin_up, stream)
    torch.cuda.synchronize()
    p0 = case.pushes()
    clocks = ClockSampler(local)
    clocks.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    case.step(args.steps, stream)
    e1.record()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    pushes = case.pushes() - p0
    _, ms_max, pushes_all = replica_throughput(dist, pushes, ms)
    status = case.status()
    resid = case.field_residual()

    # per-operator breakdown (CUDA events on the launching stream), for the roofline
    ops = {"Field": case.Field, "Move": case.Move, "SortBoundary": case.SortBoundary, "MCC": case.MCC,
           "Deposit": case.Deposit}
    reps = 3
    op_ms = {k: 0.0 for k in ops}
    move_particles = 0
    changes0 = case.slot_changes()
    t = case.tstep()
    for r in range(reps):
        case.set_tstep(t + r + 1)
        for name, fn in ops.items():
            if name == "Move":
                move_particles += sum(case.particles_count(s) for s in range(case.info.nsp))
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn(stream)
            b.record()
            torch.cuda.synchronize()
            op_ms[name] += a.elapsed_time(b) / reps
    move_bytes = (MOVE_BYTES_PER_PARTICLE * move_particles +
                  MOVE_BYTES_PER_SLOT_CHANGE * (case.slot_changes() - changes0)) / reps
    peak, peak_kind = peaks()
    achieved = move_bytes / (op_ms["Move"] * 1e-3) / 1e9
    traffic = move_traffic(args.workload)

    # end to end through the C ABI with host buffers: the initial particle
    # state comes from pinned host memory, K steps run, the time-averaged
    # densities and potential come back to host memory
    pinned = []
    for s in range(setup.info.nsp):
        counts, arrs = setup.particles(s, layout=0)
        parr = [torch.from_numpy(a).pin_memory() for a in arrs]
        pinned.append((counts, parr))
    G, nsp = case.info.Gsize, case.info.nsp
    out_den = torch.empty(nsp * G, dtype=torch.float64).pin_memory()
    out_phi = torch.empty(G, dtype=torch.float64).pin_memory()
    h2d = sum(sum(a.numel() * 4 for a in parr) + counts.nbytes for counts, parr in pinned)
    d2h = out_den.numel() * 8 + out_phi.numel() * 8
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record()
    pe0 = case.pushes()
    for s, (counts, parr) in enumerate(pinned):
        hpic._check(hpic.lib().hp_set_particles(case.h, s, counts.ctypes.data_as(hpic._I),
                                                *[hpic.C.cast(a.data_ptr(), hpic._F) for a in parr]))
    case.reset_averages()
    case.step(args.steps, stream)
    hpic.lib().hp_get_grid(case.h, hpic.GRID["AVE_DEN"], hpic.C.c_void_p(out_den.data_ptr()), d2h)
    hpic.lib().hp_get_grid(case.h, hpic.GRID["AVE_PHI"], hpic.C.c_void_p(out_phi.data_ptr()), out_phi.numel() * 8)
    f1.record()
    torch.cuda.synchronize()
    e2e_ms = allreduce(dist, f0.elapsed_time(f1), "max")
    e2e_pushes = allreduce(dist, case.pushes() - pe0, "sum")
    kernels, rooflines = kernel_rooflines(case, stream, peak, peak_kind, args.workload)

    result = dict(
        metric=METRIC, value=pushes_all / (ms_max * 1e-3), unit=UNIT, n_gpus=world, steps=args.steps,
        warmup=args.warmup, ms_per_step=ms_max / args.steps, higher_is_better=True, scaling="weak",
        vs_baseline=None, dtype="f32 particles / f64 charge and field refinement", data="synthetic",
        config=dict(workload=args.workload, nodes=f"{w['ngx']}x{w['ngy']}", ppc_per_species=w["ppc"],
                    particles=int(sum(case.particles_count(s) for s in range(nsp))),
                    gas=w.get("gas", "Ar"), pressure_torr=w["pressure"], rf_voltage=w["voltage"],
                    field_mode=case.info.field_mode,
                    parallelism=f"replicas x{world}", l2="state (>4 GB) larger than L2: no flush needed",
                    untimed_steps_before_timing=args.warmup + spin_up,
                    field_relative_residual=resid, device_status=status),
        e2e=dict(value=e2e_pushes / (e2e_ms * 1e-3), unit=UNIT, h2d_bytes_per_step=h2d / args.steps,
                 d2h_bytes_per_step=d2h / args.steps),
        roofline=dict(bound="hbm", kernel="k_move", achieved=achieved, peak=peak, unit="GB/s", frac=achieved / peak,
                      peak_source=peak_kind, traffic=traffic, algorithmic_bytes_per_launch=move_bytes),
        op_ms=op_ms,
        kernels=kernels,
        rooflines=rooflines,
        gpu_launches=case.step_kernels() * args.steps,
        clocks=clk,
    )
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        result["cpu_baseline"] = cpu_baseline(setup, case.opts)
    if rank == 0 and world == 1 and not args.no_fp64_check:
        case.close()
        result["fp64_check"] = fp64_check(stream)
        result["fp64_check_aro2"] = fp64_check(stream, "aro2_129x65_50ppc")
    return result


def run_reference(args):
    """The reference's CPU path on this host, on the same workload: its own
    set-up code (oracle/_ref/ref_dump: deck, geometry, matrix, sources,
    species, particle load; the CUDA-side set-up restated in
    oracle/refsetup.py) and the oracle's restatement of its step with its own
    numerics (PCG to its absolute tolerance, one cell crossing per push), on
    all host threads.  Nothing of this library is imported or loaded."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import refsetup
    w = WORKLOADS[args.workload]
    base = dict(metric=METRIC, unit=UNIT, impl="reference")
    if not refsetup.available():
        return dict(base, unavailable="oracle/_ref/ref_dump (the reference's set-up code) was not built")
    if w.get("gas", "Ar") != "Ar":
        return dict(base, unavailable="the reference arm's set-up covers the Ar reaction set only")
    setup = refsetup.RefSetup(json.dumps(make_deck(w)), seed=1000, field_mode=0, move_mode=0)
    budget = float(os.environ.get("HPIC_REF_BUDGET_S", "90"))
    cb = cpu_baseline(setup, setup.opts, budget_s=budget, what="the reference's set-up and step algorithm")
    return dict(base, value=cb["value"], n_gpus=int(os.environ.get("WORLD_SIZE", "1")),
                steps=args.steps, warmup=args.warmup, higher_is_better=True, scaling="weak", vs_baseline=None,
                dtype="f32", data="synthetic",
                config=dict(workload=args.workload, nodes=f"{w['ngx']}x{w['ngy']}", ppc_per_species=w["ppc"],
                            field="PCG, absolute r'z tolerance (the reference's rule)",
                            move="one cell crossing per push (the reference's rule)"),
                cpu_baseline=dict(kind=cb["kind"], cores=cb["cores"], sample=cb["sample"], value=cb["value"],
                                  unit=UNIT),
                e2e=dict(value=cb["value"], unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0))


def _setups(specs, **opts):
    """Host set-ups of many decks in parallel (the library releases the GIL)."""
    import concurrent.futures as cf

    import hpic
    with cf.ThreadPoolExecutor(min(16, os.cpu_count() or 1)) as ex:
        return list(ex.map(lambda sp: hpic.Setup(sp[0], seed=sp[1], **opts), specs))


def _timed_steps(fn, steps, stream):
    import torch
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    fn(steps, stream)
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b)


def run_batched(args):
    """Batched form: many independent Ar cases with uneven grids and particle
    counts advanced by one graph-captured launch per phase, launch shapes set
    by the autotuner; compared with the plain single-case path on the same
    cases, one case at a time, both with the batched numerics (field_mode 2)
    and with the reference's solver rule (field_mode 0: FP32 PCG to the
    absolute tolerance).  Both plain runs cross cells one by one (move_mode
    1): the reference's single wrap lets the state go non-finite within ~100
    steps at these time steps, which would time a broken run."""
    import torch

    import hpic
    from hpic.workloads import batched_cases
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream().cuda_stream
    specs = batched_cases(args.cases, seed=2024)
    opts = dict(field_mode=2, gas_temp_mode=1, move_mode=1)
    setups = _setups([(d, sd) for d, sd, _ in specs], **opts)

    def plain(field_mode, move_mode):
        pushes, ms, bad = 0, 0.0, 0
        for S, (_, sd, _) in zip(setups, specs):
            c = hpic.Case(setup=S, seed=sd, field_mode=field_mode, move_mode=move_mode, gas_temp_mode=1)
            c.step(args.warmup, stream)
            torch.cuda.synchronize()
            p0 = c.pushes()
            ms += _timed_steps(c.step, args.steps, stream)
            pushes += c.pushes() - p0
            bad += 1 if c.status() else 0
            c.close()
        return pushes / (ms * 1e-3), ms, bad

    plain2, plain2_ms, plain2_bad = plain(2, 1)
    plain0, plain0_ms, plain0_bad = plain(0, 1)
    cases = [hpic.Case(setup=S, seed=sd, **opts) for S, (_, sd, _) in zip(setups, specs)]
    batch = hpic.Batch(cases)
    t0 = time.perf_counter()
    batch.autotune(stream)
    tune_s = time.perf_counter() - t0
    batch.step(args.warmup, stream)
    torch.cuda.synchronize()
    p0 = sum(c.pushes() for c in cases)
    clocks = ClockSampler(0)
    clocks.start()
    ms = _timed_steps(batch.step, args.steps, stream)
    clk = clocks.stop()
    pushes = sum(c.pushes() for c in cases) - p0
    status = [c.status() for c in cases]
    value = pushes / (ms * 1e-3)
    res = dict(metric=METRIC, value=value, unit=UNIT, n_gpus=1, steps=args.steps, warmup=args.warmup,
               ms_per_step=ms / args.steps, higher_is_better=True, scaling="weak", vs_baseline=None,
               dtype="f32 particles / f64 charge and field refinement", data="synthetic", form="batched",
               config=dict(workload=f"batched_ar_{args.cases}cases", cases=args.cases,
                           grids="65x33/129x65/257x129", pressure_torr="10-200 mTorr log-uniform",
                           rf_voltage="50-300 V", ppc="20-200", seeds="per case",
                           particles=int(sum(sum(c.particles_count(s) for s in range(c.info.nsp)) for c in cases)),
                           tune=batch.tune(), autotune_s=round(tune_s, 2)),
               plain=dict(field_mode2_value=plain2, field_mode0_value=plain0,
                          batched_over_plain_mode2=value / plain2, batched_over_plain_reference_rule=value / plain0,
                          status_nonzero_mode2=plain2_bad, status_nonzero_reference_rule=plain0_bad,
                          note="plain = each case alone through hp_step, one after another, same steps"),
               gpu_launches=batch.step_kernels() * args.steps, clocks=clk,
               device_status_nonzero=int(sum(1 for x in status if x)),
               device_status_bits={f"0x{b:x}": int(sum(1 for x in status if x & b)) for b in (1, 2, 4, 8, 16)},
               device_status_cases=[dict(specs[k][2], status=int(status[k])) for k in range(len(cases)) if status[k]])
    batch.close()
    for c in cases:
        c.close()
    return res


def run_served(args):
    """Served form: a Poisson stream of requests (Ar CCPs of every grid size,
    1-10 RF periods each, scaled by --steps-scale) through the request loop,
    against the same stream served one case at a time on the plain path."""
    import torch

    import hpic
    from hpic.workloads import served_stream
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream().cuda_stream
    steps_per_cycle = max(1, int(round(400 * args.steps_scale)))
    reqs = served_stream(args.requests, rate_per_s=args.rate, seed=7, steps_per_cycle=steps_per_cycle)
    # initial particles generated on the device unless --host-load (both loops alike)
    opts = dict(field_mode=2, gas_temp_mode=1, move_mode=1, gpu_load=0 if args.host_load else 1)

    def pct(v, q):
        return float(np.percentile(np.asarray(v), q)) if v else None

    # the request loop
    srv = hpic.Server(max_slots=args.slots, steps_per_launch=args.steps_per_launch,
                      mem_budget_bytes=int(args.budget_gb * (1 << 30)), **opts)
    t_start = time.perf_counter()
    arrival_clock = {}
    k, results = 0, []
    while k < len(reqs) or len(results) < len(reqs):
        now = time.perf_counter() - t_start
        while k < len(reqs) and reqs[k][0] <= now:
            _, deck, nsteps, seed, _ = reqs[k]
            arrival_clock[srv.submit(deck, nsteps, seed)] = reqs[k][0]
            k += 1
        pending = srv.poll(stream)
        results += srv.results()
        if pending == 0 and k < len(reqs):
            time.sleep(max(0.0, min(0.05, reqs[k][0] - (time.perf_counter() - t_start))))
    t_end = time.perf_counter() - t_start
    srv.close()
    lat = [r.t_done - r.t_submit for r, _, _ in results if r.error == 0]
    pushes = sum(r.particle_pushes for r, _, _ in results)
    errors = sum(1 for r, _, _ in results if r.error)
    status_nonzero = sum(1 for r, _, _ in results if r.error == 0 and r.status)
    status_bits = {f"0x{b:x}": int(sum(1 for r, _, _ in results if r.error == 0 and r.status & b))
                   for b in (1, 2, 4, 8, 16, 32)}
    # the same stream, one case at a time on the plain path (set-up included);
    # --plain-requests bounds it to the stream's first requests
    n_plain = len(reqs) if args.plain_requests <= 0 else min(args.plain_requests, len(reqs))
    t_start = time.perf_counter()
    plain_lat, plain_pushes = [], 0
    for t_arr, deck, nsteps, seed, _ in reqs[:n_plain]:
        now = time.perf_counter() - t_start
        if now < t_arr:
            time.sleep(t_arr - now)
        c = hpic.Case(deck, seed=seed, **opts)
        c.step(nsteps, stream)
        n = c.average_count()
        _ = c.grid("AVE_DEN") / n, c.grid("AVE_PHI") / n
        plain_pushes += c.pushes()
        c.close()
        plain_lat.append(time.perf_counter() - t_start - t_arr)
    plain_end = time.perf_counter() - t_start
    value = pushes / t_end
    return dict(metric=METRIC, value=value, unit=UNIT, n_gpus=1, steps=None, warmup=0, higher_is_better=True,
                scaling="weak", vs_baseline=None, dtype="f32 particles / f64 charge and field refinement",
                data="synthetic", form="served",
                config=dict(workload=f"served_ar_{args.requests}req", requests=args.requests,
                            arrivals=f"Poisson {args.rate}/s", grids="65x33/129x65/257x129/513x257",
                            ppc="50-200", rf_periods="1-10", steps_per_rf_period=steps_per_cycle,
                            slots=args.slots, steps_per_launch=args.steps_per_launch, budget_gb=args.budget_gb,
                            gas="Ar or 80/20 Ar/O2", particle_load="host" if args.host_load else "device"),
                latency_s=dict(p50=pct(lat, 50), p99=pct(lat, 99)), errors=errors,
                device_status_nonzero=status_nonzero, device_status_bits=status_bits, wall_s=t_end,
                plain=dict(value=plain_pushes / plain_end, latency_s=dict(p50=pct(plain_lat, 50),
                                                                          p99=pct(plain_lat, 99)),
                           requests=n_plain, wall_s=plain_end, served_over_plain=value / (plain_pushes / plain_end)))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="ar_513x257_200ppc", choices=list(WORKLOADS))
    ap.add_argument("--field-mode", type=int, default=2)
    ap.add_argument("--move-mode", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64-check", action="store_true")
    ap.add_argument("--form", default="single", choices=["single", "batched", "served"],
                    help="single: the large case (default); batched: --cases mixed cases in one batch; "
                         "served: a request stream through hp_server")
    ap.add_argument("--cases", type=int, default=64)
    ap.add_argument("--requests", type=int, default=64)
    ap.add_argument("--rate", type=float, default=4.0)
    ap.add_argument("--steps-scale", type=float, default=0.1, help="served: steps per RF period / 400")
    ap.add_argument("--plain-requests", type=int, default=0,
                    help="served: the plain arm runs the stream's first N requests (0: all)")
    ap.add_argument("--slots", type=int, default=64)
    ap.add_argument("--steps-per-launch", type=int, default=40)
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--host-load", action="store_true",
                    help="served: load the initial particles on the host (the reference's loader) instead of the device")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank = int(os.environ.get("RANK", "0"))
    if args.form != "single" and args.impl == "ours":
        if rank == 0:
            res = run_batched(args) if args.form == "batched" else run_served(args)
            print(json.dumps(res), flush=True)
        return
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    rank, world, local, dist = dist_init(args.gpus)
    res = run_ours(args, rank, world, local, dist)
    if rank == 0:
        print(json.dumps(res), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
