"""Benchmark of the RELAX relaxation step on B200.

Workload: power-law (n = 3) relaxation under a 20-degree thrust with one
rate-strengthening afterslip plane, FFT box 256 x 256 x 128 (dx = 0.5 km),
adaptive time step -- synthetic, seeded input of the named configuration
(relax_b200.config.powerlaw_thrust).  A "step" is one RK2
predictor/corrector step of RELAX's time loop (src/relax.f90:555-890).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line.  value = grid points x steps / s over all ranks
(replicas: every rank advances its own instance; no data-path collective).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "grid-pt*RK2-steps/s"
UNIT = "grid-pt*steps/s"


def workload():
    from relax_b200.config import powerlaw_thrust
    return powerlaw_thrust(sx=256, sz=128, dx=0.5)


def config_desc(sim):
    return {
        "workload": f"power-law n=3 thrust + afterslip plane, box {sim.sx1}x{sim.sx2}x{sim.sx3}, "
                    f"dx={sim.dx1} km, adaptive dt",
        "grid": [sim.sx1, sim.sx2, sim.sx3],
        "grid_points": sim.npoints,
        "afterslip_planes": len(sim.planes),
        "l2": "inputs larger than L2: ~0.7 GB device working set per step (126 MB L2)",
        "parallelism": "replicas",
    }


# --------------------------------------------------------------------------
# clocks during the timed region
# --------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
                except ValueError:
                    continue
        os.unlink(self.path)
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for _, _, r in rows for k in range(4) if r[k].lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "samples": len(rows), "reasons": reasons}


# --------------------------------------------------------------------------
# algorithmic bytes per launch of each kernel: every operand of the stage
# streamed once in FP32
# --------------------------------------------------------------------------
def kernel_bytes(sim):
    sx1, sx2, sx3 = sim.sx1, sim.sx2, sim.sx3
    h = sx3 // 2
    nh = sx1 * sx2 * h
    K1 = sx1 // 2 + 1
    spec_plane = 3 * sx2 * K1 * 8          # one x3-plane of the 3-component spectrum
    return {
        # tau, m, u in; tau, m out (sig is stored only on the afterslip bands)
        "k_stress<END>": nh * (24 + 24 + 12 + 24 + 24),
        # m, tau, v, gamma in; m, gamma out
        "k_stress<CORR>": nh * (24 + 24 + 12 + 4 + 24 + 4),
        # moment in, spectrum (body planes + traction plane) out
        "k_xfwd": nh * 24 + (h + 1) * spec_plane,
        "k_ypass<fwd>": 2 * (h + 1) * spec_plane,
        # body planes + traction plane in, body planes out
        "k_zspec": (h + 1) * spec_plane + h * spec_plane,
        "k_ypass<inv>": 2 * h * spec_plane,
        # spectrum + base field in, field out
        "k_xinv": h * spec_plane + nh * 12 + nh * 12,
    }


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_from_profiles():
    """dram read+write bytes per launch of the dominant kernel, from the
    committed ncu summary (scaled to the benchmark grid), or None."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


# --------------------------------------------------------------------------
# the CPU oracle (reported baseline, reference arm)
# --------------------------------------------------------------------------
def cpu_sample(sim, nsteps: int):
    """Times RK2 steps 2..nsteps of the oracle (FP32 restatement of the
    reference CPU path) on the host cores; returns (rate, cores, seconds)."""
    import ctypes as C
    from oracle.oracle import Oracle
    from relax_b200.config import relax_step_log
    o = Oracle(32)
    cfg, keep = sim.to_c(o.structure_fn)
    st = o.lib.orc_state_create(C.byref(cfg))
    lg = relax_step_log()
    try:
        o.lib.orc_coseismic(st, C.byref(lg))
        o.lib.orc_step(st, None, C.byref(lg))          # step 1 untimed
        t0 = time.perf_counter()
        for _ in range(nsteps):
            rc = o.lib.orc_step(st, None, C.byref(lg))
            assert rc == 0
        dt = time.perf_counter() - t0
    finally:
        o.lib.orc_state_free(st)
    return sim.npoints * nsteps / dt, o.threads(), dt


def rel_l2(a, b):
    import numpy as np
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    nb = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def accuracy_vs_fp64(sim, nsteps: int, device: int, mixed: bool):
    """The checker half of the CPU leg (untimed): the workload stepped
    nsteps times on the GPU through the public API from a fresh context in
    the plain FP32 form (adaptive Dt) and, when `mixed`, in the
    mixed-precision form with the plain run's Dt sequence prescribed; the
    FP64 oracle (every field in double precision, the same method) replays
    that Dt sequence.  Relative L2 of each field after the run (u over the
    physical half-space without the two pad columns)."""
    import numpy as np
    from oracle.oracle import Oracle
    from relax_b200.api import Relax
    t0 = time.perf_counter()

    def gpu(mode, dts=None):
        with Relax(sim, device=device) as r:
            if mode == "mixed":
                r.set_precision("mixed")
            logs = [r.coseismic()]
            for k in range(nsteps):
                logs.append(r.step(None if dts is None else dts[k]))
            return logs, {k: r.field(k) for k in ("u", "sig", "tau", "gamma")}

    logs, g = gpu("fp32")
    dts = [lg[1] for lg in logs[1:]]
    runs = {"fp32": (logs, g)}
    if mixed:
        runs["mixed"] = gpu("mixed", dts)
    rlogs, ref = Oracle(64).run(sim, nsteps, dt_schedule=dts)

    def tens(t):
        return np.stack([t[n].astype(np.float64) for n in t.dtype.names], axis=-1)

    out = {"vs": "FP64 oracle (oracle/relax_oracle.c built with every field in double precision), "
                 "replaying the plain run's Dt sequence",
           "steps": nsteps, "bound": 1e-4}
    for name, (lg, f) in runs.items():
        err = {"u": rel_l2(f["u"][..., :-2], ref["u"][..., :-2]),
               "sig": rel_l2(tens(f["sig"]), tens(ref["sig"])),
               "tau": rel_l2(tens(f["tau"]), tens(ref["tau"])),
               "gamma": rel_l2(f["gamma"][..., :-2], ref["gamma"][..., :-2])}
        logdev = {q: max(abs(a[c] - b[c]) / abs(b[c]) for a, b in zip(lg[1:], rlogs[1:]) if b[c] != 0)
                  for q, c in (("power", 6), ("cei", 7))}
        out[name] = {"rel_l2": err, "within_bound": max(err.values()) <= 1e-4, "log_rel_dev": logdev}
    out["seconds"] = round(time.perf_counter() - t0, 1)
    return out


def max_over_ranks(v: float, dist=None, device: str = "cpu") -> float:
    """The largest value over the ranks of the process group (every rank
    takes the same collective step); v itself without a group."""
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference(args, rank, world):
    sim = workload()
    if rank != 0:
        return 0
    # each reference step is one full oracle RK2 step of the workload; the
    # run is bounded to a few minutes of host time
    t0 = time.perf_counter()
    rate1, cores, dt1 = cpu_sample(sim, 1)
    per_step = dt1
    budget = 150.0
    k = max(1, min(args.steps, int(budget / max(per_step, 1e-3)) - 1))
    rate, cores, dt = cpu_sample(sim, k)
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": world,
        "steps": k, "warmup": 1, "ms_per_step": 1e3 * dt / k, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config_desc(sim),
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{k} RK2 steps of the full {sim.sx1}x{sim.sx2}x{sim.sx3} "
                                   "workload after the coseismic solve and one untimed step "
                                   "(the reference cannot be compiled here; the oracle restates "
                                   "its CPU path)"},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": time.perf_counter() - t0,
    }
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------
# the B200 arm
# --------------------------------------------------------------------------
def run_gpu(args, rank, world, local_rank):
    import torch
    from relax_b200.api import Relax

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
    sim = workload()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def allmax(v):
        return max_over_ranks(v, dist, "cuda")

    import ctypes as C

    def timed_form(mode, wsim=sim, steps=None, warmup=None):
        """W warm-up steps, then K steps timed with CUDA events on the
        context's stream (barrier + synchronize on both sides), then a
        profiled pass of per-kernel durations."""
        steps = args.steps if steps is None else steps
        warmup = args.warmup if warmup is None else warmup
        r = Relax(wsim, device=local_rank)
        if mode == "mixed":
            r.set_precision("mixed")
        r.coseismic()
        for _ in range(warmup):
            r.step()
        s = C.c_void_p()
        r.lib.relax_get_stream(r.h, C.byref(s))
        stream = torch.cuda.ExternalStream(s.value)
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        clk = ClockSampler(local_rank)
        clk.start()
        time.sleep(0.3)
        barrier()
        n0 = r.launch_count()
        ev0.record(stream)
        for _ in range(steps):
            lg = r.step()
            if lg[0] == 0:
                raise RuntimeError("simulation ended inside the timed region")
        ev1.record(stream)
        barrier()
        launches = r.launch_count() - n0
        ms = ev0.elapsed_time(ev1)
        clocks = clk.stop()
        ms = allmax(ms)
        # per-kernel durations (CUDA events around each launch, separate pass)
        r.profile(True)
        nprof = max(3, min(steps, 10))
        for _ in range(nprof):
            r.step()
        prof = r.profile_read()
        r.profile(False)
        r.close()
        return ms, launches, clocks, prof, nprof

    ms, launches, clocks, prof, nprof = timed_form("fp32")
    ms_step = ms / args.steps
    value = world * sim.npoints * args.steps / (ms / 1e3)
    algo = kernel_bytes(sim)
    kernels = {}
    for name, (tot, n) in prof.items():
        d = {"ms_total": tot, "launches": n, "ms_per_launch": tot / n}
        if name in algo:
            d["alg_bytes"] = algo[name]
            d["gbs"] = algo[name] / (tot / n / 1e3) / 1e9
        kernels[name] = d
    step_ms_prof = sum(v[0] for v in prof.values()) / nprof
    dom = max((k for k in kernels if k in algo), key=lambda k: kernels[k]["ms_total"])
    peak, peak_kind = peaks()
    ach = kernels[dom]["gbs"]
    traffic = traffic_from_profiles().get(dom)

    # the large single instance (512^2 x 256 box, gravity, three seeded
    # faults, n = 3.5 below a 25 km lid): a few steps, plain form
    large = None
    if not args.no_large:
        from relax_b200.config import random_faults
        lsim = random_faults(1)
        lsteps = 5
        lms, llaunches, lclocks, lprof, lnprof = timed_form("fp32", lsim, lsteps, 3)
        lstep = lms / lsteps
        lb = 536.0 * lsim.npoints
        lalgo = kernel_bytes(lsim)
        lk = {}
        for name, (tot, n) in lprof.items():
            d = {"ms_per_launch": tot / n, "launches": n}
            if name in lalgo:
                d["gbs"] = lalgo[name] / (tot / n / 1e3) / 1e9
            lk[name] = d
        large = {"workload": f"random faults seed 1, box {lsim.sx1}x{lsim.sx2}x{lsim.sx3}, dx={lsim.dx1} km, "
                             "gravity 8.3e-4, n=3.5 below 25 km, adaptive dt",
                 "grid_points": lsim.npoints, "steps": lsteps, "warmup": 3,
                 "value": world * lsim.npoints * lsteps / (lms / 1e3), "unit": UNIT, "ms_per_step": lstep,
                 "step_roofline": {"alg_bytes_per_step": lb, "achieved_gbs": lb / (lstep / 1e3) / 1e9,
                                   "frac": lb / (lstep / 1e3) / 1e9 / peaks()[0]},
                 "kernels": lk, "gpu_launches": llaunches, "clocks": lclocks}

    # the linear Maxwell configuration (128^2 x 128 box, Dt = 0.5): 20 steps
    # timed after 3 warm-up steps, plain form (the interval also holds the
    # 10 profiled steps that follow)
    from relax_b200.config import linear_maxwell
    csim = linear_maxwell(sx=128, sz=128, dx=0.8, steps=33)
    cms, claunches, cclocks, _, _ = timed_form("fp32", csim, 20, 3)
    cstep = cms / 20
    c1 = {"workload": "linear Maxwell below 30 km, vertical strike-slip fault, box 128x128x128, dx=0.8 km, "
                      "Dt=0.5, 20 timed steps",
          "grid_points": csim.npoints, "steps": 20, "warmup": 3,
          "value": world * csim.npoints * 20 / (cms / 1e3), "unit": UNIT, "ms_per_step": cstep,
          "step_roofline": {"alg_bytes_per_step": 536.0 * csim.npoints,
                            "achieved_gbs": 536.0 * csim.npoints / (cstep / 1e3) / 1e9,
                            "frac": 536.0 * csim.npoints / (cstep / 1e3) / 1e9 / peaks()[0]},
          "gpu_launches": claunches, "clocks": cclocks}

    # the mixed-precision form beside the plain one (x3 transform's DFT-64
    # sub-transforms on the tensor cores), same workload, same timing
    mixed = None
    if sim.sx3 == 128:
        mms, mlaunches, mclocks, mprof, mnprof = timed_form("mixed")
        mvalue = world * sim.npoints * args.steps / (mms / 1e3)
        mk = {}
        for name, (tot, n) in mprof.items():
            d = {"ms_total": tot, "launches": n, "ms_per_launch": tot / n}
            if name in algo:
                d["alg_bytes"] = algo[name]
                d["gbs"] = algo[name] / (tot / n / 1e3) / 1e9
            mk[name] = d
        mixed = {"value": mvalue, "unit": UNIT, "ms_per_step": mms / args.steps,
                 "speedup_vs_plain": mvalue / value, "gpu_launches": mlaunches, "clocks": mclocks,
                 "kernel_ms_per_step": sum(v[0] for v in mprof.values()) / mnprof,
                 "k_zspec": mk.get("k_zspec"),
                 "form": "x3 transform as two interleaved length-64 DFTs per column, each a tcgen05 "
                         "BF16 product with hi/lo split operands (3 products) and FP32 accumulation; "
                         "everything else as the plain form"}

    # end to end through the public API with host buffers: create (H2D of the
    # deck, structures and prestress), coseismic solve, K steps each reading
    # back its log record, D2H of the displacement and stress fields into
    # page-locked host buffers the caller allocated beforehand
    ushape = sim.vec_shape()
    u = torch.empty(ushape[0] * ushape[1] * ushape[2] * ushape[3], dtype=torch.float32,
                    pin_memory=True).numpy().reshape(ushape)
    tau = torch.empty(sim.npoints // 2 * 6, dtype=torch.float32, pin_memory=True).numpy()
    # five passes, the median reported (set-up times vary with the state of
    # the device memory allocator)
    passes = []
    for _ in range(5):
        barrier()
        t0 = time.perf_counter()
        r2 = Relax(sim, device=local_rank)
        r2.coseismic()
        for _ in range(args.steps):
            r2.step()
        r2.field_into("u", u)
        r2.field_into("tau", tau)
        r2.close()
        torch.cuda.synchronize()
        passes.append(allmax(time.perf_counter() - t0))
    e2e_s = statistics.median(passes)
    nz = sim.sx3h
    # H2D: the deck's per-depth structures and the twiddle tables (the
    # prestress is filled on the device from its per-depth values)
    h2d = (64 * 6 * nz * 3 + 8 * (sim.sx1 // 2 + sim.sx1 + sim.sx2 + sim.sx3)) / args.steps
    d2h = 120 + (u.nbytes + tau.nbytes) / args.steps
    e2e = {"value": world * sim.npoints * args.steps / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
           "timing": "host wall clock around create + coseismic + K steps + field readback, "
                     "median of 5 passes",
           "passes_s": [round(x, 4) for x in passes]}

    if rank != 0:
        return 0
    # the two ensembles, 10 steps each after the tuning steps, on rank 0's GPU
    ens = {}
    if world == 1 and not args.no_ensemble:
        for which in ("c4", "c5"):
            ens[which] = ensemble_figure(which, 10, 6, local_rank)
    cpu = None
    accuracy = None
    if world == 1 and not args.no_cpu:
        rate, cores, dt = cpu_sample(sim, 2)
        cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": "2 RK2 steps of the same workload on the host cores (after the "
                         "coseismic solve and one untimed step), FP32 oracle restating the "
                         "reference CPU path"}
        accuracy = accuracy_vs_fp64(sim, args.steps, local_rank, mixed is not None)
        # the other named single-instance configurations against the FP64
        # oracle: the linear Maxwell box for its full 20 steps, and the large
        # instance for one step (the oracle takes about a minute per step there)
        from relax_b200.config import linear_maxwell, random_faults
        accuracy["C1"] = accuracy_vs_fp64(linear_maxwell(sx=128, sz=128, dx=0.8, steps=20), 20, local_rank,
                                          False)
        if not args.no_large:
            accuracy["C3"] = accuracy_vs_fp64(random_faults(1), 1, local_rank, False)
    b_alg = 536.0 * sim.npoints
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config_desc(sim),
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak,
                     "unit": "GB/s", "frac": ach / peak, "peak_kind": peak_kind,
                     "traffic": traffic},
        "step_roofline": {"alg_bytes_per_step": b_alg,
                          "achieved_gbs": b_alg / (ms_step / 1e3) / 1e9,
                          "frac": b_alg / (ms_step / 1e3) / 1e9 / peak,
                          "note": "536 B per grid point per RK2 step of the reference data flow; "
                                  "the fused kernels move less than that"},
        "kernels": kernels,
        "kernel_ms_per_step": step_ms_prof,
        "gpu_launches": launches,
        "clocks": clocks,
        "e2e": e2e,
        "cpu_baseline": cpu,
        "accuracy": accuracy,
        "mixed": mixed,
        "large_instance": large,
        "c1_instance": c1,
        "ensemble_c4": ens.get("c4"),
        "ensemble_c5": ens.get("c5"),
    }
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------
# the batched ensemble (64 members, uneven grids), against a loop of plain solves
# --------------------------------------------------------------------------
def ensemble_figure(which: str, K: int, W: int, device: int = 0):
    """K ensemble steps (after W warm-up steps) of every member through
    relax_ensemble (one batch per grid shape, each on its own stream, one
    host synchronisation per step) against the same members solved one
    after the other through relax_step; host wall clock around the K steps,
    the device synchronised on both sides."""
    import collections
    import torch
    from relax_b200.api import Ensemble, Relax
    from relax_b200.config import ensemble_uneven

    if which == "c5":
        from relax_b200.config import ensemble_thrust_afterslip
        sims = ensemble_thrust_afterslip(seed=5, n=16)
        workload_name = ("16 thrust instances on 256^2x128 (dx 0.5 km, gravity), 5 km slip patches "
                         "2(1+N(0,0.2)), two afterslip planes, n=3 below 35 km")
    else:
        sims = ensemble_uneven(seed=4, n=64)
        workload_name = ("uneven ensemble of 64 members, grids {64^3, 128^2x64, 128^3, 192^2x96}, "
                         "power-law n U[1,3.5], prefactor 10^U[-1,1], lid U[15,40] km, one fault each")
    shapes = collections.Counter((s.sx1, s.sx2, s.sx3) for s in sims)
    npts = sum(s.npoints for s in sims)
    # each shape group tunes itself on its first six steps (batched launches
    # against the members in turn): the warm-up covers them
    W = max(W, 6)

    with Ensemble(sims, device) as e:
        e.coseismic()
        for _ in range(W):
            e.step()
        n0 = e.launch_count()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(K):
            e.step()             # ends with the ensemble's host synchronisation
        torch.cuda.synchronize()
        t_batch = time.perf_counter() - t0
        launches = e.launch_count() - n0
        groups = e.groups()
        tuning = {"%dx%dx%d" % g["grid"]: {"members": g["members"], "mode": g["mode"],
                                           "batched_ms": round(g["batched_ms"], 4),
                                           "in_turn_ms": round(g["in_turn_ms"], 4)} for g in e.tuning()}

    # the loop of plain solves: each member alone through relax_step
    t_loop = 0.0
    per_shape_loop = collections.Counter()
    for s in sims:
        with Relax(s, device) as r:
            r.coseismic()
            for _ in range(W):
                r.step()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(K):
                r.step()
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
            t_loop += dt
            per_shape_loop[(s.sx1, s.sx2, s.sx3)] += dt

    steps_per_solve = 100
    solves = len(sims) * K / steps_per_solve
    return {
        "metric": "ensemble solves/s (100 RK2 steps per member)", "value": solves / t_batch,
        "unit": "solves/s", "steps": K, "warmup": W, "higher_is_better": True,
        "workload": workload_name, "members": {f"{a}x{b}x{c}": n for (a, b, c), n in shapes.items()},
        "groups": groups, "grid_points_total": npts, "tuning": tuning,
        "timing": "host wall clock around K ensemble steps (one host synchronisation each), after W warm-up steps "
                  "(at least the six steps of each group's tuning)",
        "grid_pt_steps_per_s": npts * K / t_batch,
        "loop_of_plain_solves": {"value": solves / t_loop, "unit": "solves/s",
                                 "grid_pt_steps_per_s": npts * K / t_loop,
                                 "ms_per_step_by_shape": {f"{a}x{b}x{c}": 1e3 * v / K
                                                          for (a, b, c), v in per_shape_loop.items()}},
        "speedup_vs_loop": t_loop / t_batch,
        "gpu_launches": launches,
    }


def run_ensemble(args):
    import torch
    torch.cuda.set_device(0)
    fig = ensemble_figure(args.ensemble, args.steps, args.warmup)
    line = {"metric": fig["metric"], "value": fig["value"], "unit": fig["unit"], "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": fig["workload"], "members": fig["members"], "parallelism": "one batch per shape",
                       "timing": fig["timing"]},
            "ensemble": fig, "gpu_launches": fig["gpu_launches"]}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-large", action="store_true", help="skip the 512^2 x 256 single-instance figure")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the ensemble figures of the default line")
    ap.add_argument("--ensemble", nargs="?", const="c4", choices=["c4", "c5"], default=None,
                    help="a batched ensemble against a loop of plain solves (1 GPU): c4, the 64 uneven "
                         "members (default), or c5, 16 thrust instances with afterslip")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    if args.ensemble:
        return run_ensemble(args)
    try:
        if args.impl == "reference":
            rc = run_reference(args, rank, world)
        else:
            rc = run_gpu(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    return rc


if __name__ == "__main__":
    sys.exit(main())
