#!/usr/bin/env python
"""Benchmark of the B200 CUEVA hot path: zone-updates/s of the resistive
relativistic MHD Kelvin-Helmholtz run (plain FP64 and mixed precision).

Workload: 2048 x 4096 cells, MP5 + HLLC, IMEX SSP3(4,3,3), sigma = 1e6
(synthetic KH initial data, reference orientation), the resistive KH run the
metric is quoted on.  One bench "step" is one full time step (4 RK stages) of
that grid; the state stays resident in HBM.
`e2e` repeats the measurement through the C-ABI with host buffers: each step
uploads the 14 primitive fields from pinned host memory, advances one step
and downloads them again, all inside the timed region (the readback of step k
overlaps the upload of step k+1 field by field; the synchronous loop is
reported beside it).

Multi-GPU: the path does not shard (one grid per GPU, no exchange), so N GPUs
run N independent replicas (weak scaling, whole-job value = N x per-replica
work / max-over-ranks time).

--impl reference times the CPU restatement of the reference on the host cores
(the Fortran reference cannot be built here: no Fortran compiler).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "mhd-kh-instability_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

METRIC = "zone-updates/s per RK step: plain FP64 vs mixed+learned C2P at L1 err<=1e-6"
UNIT = "zone-updates/s"


def alg_bytes_per_zone(s):
    """Algorithmic HBM bytes per zone-update: the 14 carried doubles in and
    out, the 17-double stage right-hand side per stage and the re-read of all
    earlier stage right-hand sides: 8 * (48 s + 8.5 s (s-1) + 28)."""
    return 8.0 * (48 * s + 8.5 * s * (s - 1) + 28)


FACE_BYTES = 8.0 * (20 + 14)   # per interface: 20 reconstructed fields read once, 14 fluxes written


def stage_kernels(cfg, s, kms, kcnt):
    """The stage kernels of the profiled steps: name -> (units per launch,
    algorithmic bytes per unit, summed ms, launches).  Slot 1 of the profile
    is the kernel that updates the points: the fused k_stage (no y-face
    launches in slot 0), or k_xupd after k_yface.  The fused kernel's bytes
    per point are the stage's share of the whole-step figure, B_alg(s) / s;
    the split kernels add the y-flux round trip and the twice-staged
    stencil fields, which the fused kernel does not move."""
    pts = (cfg.imax + 1) * (cfg.jmax + 1)
    if kcnt[0] == 0:
        return {"k_stage": (pts, alg_bytes_per_zone(s) / s, kms[1], kcnt[1])}
    return {"k_yface": ((cfg.imax + 1) * (cfg.jmax + 2), FACE_BYTES, kms[0], kcnt[0]),
            "k_xupd": (pts, 8.0 * (20 + 14) + alg_bytes_per_zone(s) / s, kms[1], kcnt[1])}


# FP64 arithmetic of the B200: 64 FP64 lanes per SM and clock on 148 SMs
# (NVIDIA's 37 TFLOP/s FP64 figure is this at 1965 MHz with an FMA counted as
# two flops).  A spec value, not measured on this pool.
FP64_LANES_PER_SM = 64
N_SM = 148


def fp64_roofline(kernels, name, sm_mhz):
    """FP64 roofline of kernel `name`: counted FP64 instructions and flops per
    unit (profiles/fp64_ops.json, from an ncu count of the same kernels)
    times the units of a launch over the launch's average CUDA-event time,
    against the FP64 lanes at the SM clock sampled during the timed region."""
    path = os.path.join(ROOT, "profiles", "fp64_ops.json")
    if not os.path.exists(path) or not sm_mhz:
        return None
    with open(path) as f:
        ops = json.load(f)
    k = ops.get("kernels", {}).get(name)
    if not k or not kernels.get(name, {}).get("avg_ms"):
        return None
    units = kernels[name]["units"]
    sec = kernels[name]["avg_ms"] * 1e-3
    instr_rate = k["fp64_instr_per_unit"] * units / sec
    flop_rate = k["fp64_flops_per_unit"] * units / sec
    lane_rate = FP64_LANES_PER_SM * N_SM * sm_mhz * 1e6
    return {"bound": "fp64", "achieved": flop_rate / 1e12, "peak": 2 * lane_rate / 1e12, "unit": "TFLOP/s",
            "frac": flop_rate / (2 * lane_rate), "pipe_frac": instr_rate / lane_rate, "kernel": name,
            "fp64_instr_per_unit": k["fp64_instr_per_unit"], "fp64_flops_per_unit": k["fp64_flops_per_unit"],
            "peak_kind": f"spec: {FP64_LANES_PER_SM} FP64 lanes/SM x {N_SM} SMs at the sampled {sm_mhz:.0f} MHz",
            "note": "frac = counted FP64 flops (FMA = 2) over the lanes' FMA peak; pipe_frac = FP64 "
                    "instructions over the lanes' issue rate (the no-FMA build keeps a multiply-add as two "
                    "instructions); counts from " + ops.get("source", "profiles/fp64_ops.json")}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None
        self.thread = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        self.n0 = 0
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # the timed region starts once the sampler reports: a short
            # region would otherwise end before nvidia-smi's first line
            t0 = time.time()
            while not self.samples and time.time() - t0 < 5.0 and self.proc.poll() is None:
                time.sleep(0.01)
            self.n0 = len(self.samples)
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc is not None:
            # one more line after the region, so a region shorter than the
            # sampling period still has a sample at its end
            n1, t0 = len(self.samples), time.time()
            while len(self.samples) <= n1 and time.time() - t0 < 2.0 and self.proc.poll() is None:
                time.sleep(0.01)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=2)

    def summary(self):
        region = self.samples[self.n0:] or self.samples
        if not region:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = sorted(float(s[1]) for s in region if s[1].replace(".", "").isdigit())
        mx = max((float(s[2]) for s in region if s[2].replace(".", "").isdigit()), default=None)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in region for k in range(4) if s[5 + k].lower() == "active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(region)}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(ms, pg, device="cuda"):
    """The largest of the ranks' device times (every rank takes part); ms
    itself without a process group."""
    if pg is None:
        return ms
    import torch
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(world, zones, steps, ms):
    """Whole-job zone-updates/s: every replica advances its own grid of
    `zones` cells `steps` times; the job takes the slowest replica's ms."""
    return world * zones * steps / (ms * 1e-3)


def cpu_port_rate(cfg, steps_budget_s=20.0, max_steps=2, threads=None, warmup=1):
    """Zone-updates/s of the CPU restatement (the oracle) on a bounded sample
    of the workload: the full grid, after `warmup` untimed steps as many whole
    steps as fit the budget (at least one, at most max_steps)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py
    oracle_py.build()
    threads = threads or os.cpu_count() or 1
    oracle_py.set_threads(threads)
    kw = cfg.solver_kwargs()
    kw.pop("precision", None)
    o = oracle_py.Oracle(**kw)
    o.set_prims(oracle_py.kh_init(cfg.imax, cfg.jmax, **{k: v for k, v in cfg.kh_kwargs().items()}))
    for _ in range(max(warmup, 1)):
        o.step(1)     # warm-up (page faults of the working set)
    n, t0 = 0, time.perf_counter()
    while n < max_steps:
        o.step(1)
        n += 1
        if time.perf_counter() - t0 > steps_budget_s:
            break
    dt = time.perf_counter() - t0
    return cfg.nx * cfg.ny * n / dt, threads, f"{n} full step(s) of the {cfg.nx}x{cfg.ny} grid ({dt:.1f} s)"


def run_reference(args, cfg):
    """The reference arm: the CPU restatement of the Fortran (the Fortran
    itself cannot be compiled here) on all host cores, same workload and
    metric.  Its steps are whole time steps of the same grid; they are
    bounded to about 90 s of CPU work, so a long --steps run stops early and
    says so in `sample`."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    value, threads, sample = cpu_port_rate(cfg, steps_budget_s=90.0, max_steps=max(args.steps, 1), threads=threads,
                                           warmup=1)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * cfg.nx * cfg.ny / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": f"synthetic KH initial data ({cfg.nx} x {cfg.ny} shear layer, reference orientation)",
            "config": {"workload": cfg.name, "nx": cfg.nx, "ny": cfg.ny, "rk_stages": 4, "solver": "MP5+HLLC",
                       "sigma": cfg.sigma},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": sample + " after 1 untimed step, bounded to ~90 s; CPU restatement of "
                                                "the Fortran (no Fortran compiler on this image)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


PRIM_NAMES = ["rho", "p", "vx", "vy", "vz", "psi", "phi", "Ex", "Ey", "Ez", "Bx", "By", "Bz", "q"]


def vector_rel_l1(run, ref):
    """Per-component L1 difference relative to the L1 norm of the whole
    vector (|v|, |E|, |B|); components that are zero in the 2D problem, or
    small against their vector, are then measured against the physics.
    `run` is a Cueva run or a dict of its fields."""
    import numpy as np
    get = run.interior if hasattr(run, "interior") else run.__getitem__
    groups = {"v": ("vx", "vy", "vz"), "E": ("Ex", "Ey", "Ez"), "B": ("Bx", "By", "Bz")}
    out = {}
    for comps in groups.values():
        den = max(float(sum(np.abs(ref[c]).sum() for c in comps)), 1e-300)
        for c in comps:
            out[c] = float(np.abs(get(c) - ref[c]).sum()) / den
    return out


def mixed_study(args):
    """Mixed precision (FP32 reconstruction + Riemann, FP64 update, implicit
    E and con2prim) against plain FP64 on the 2048x4096 V0 = 0.8, sigma = 1e5
    workload, MP7 and MP9: per-variable relative L1 after 1, 100 and 1000
    steps, and the step time of both forms."""
    import dataclasses
    import torch
    from cueva import Cueva
    from cueva.configs import C3
    from cueva.metrics import rel_l1_field
    checkpoints = [int(c) for c in args.study_steps.split(",")]
    cfg = C3
    if args.grid:
        nx, ny = (int(v) for v in args.grid.lower().split("x"))
        cfg = dataclasses.replace(C3, nx=nx, ny=ny, name=C3.name.replace("2048x4096", f"{nx}x{ny}"))
    out = {"study": "mixed precision vs plain FP64", "workload": cfg.name, "nx": cfg.nx, "ny": cfg.ny,
           "checkpoints": checkpoints, "variants": {}}
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    for rec, label in ((1, "MP7"), (2, "MP9")):
        runs = {}
        for prec in (0, 1):
            g = Cueva(pinned=False, **dict(cfg.solver_kwargs(), rec_mp=rec, precision=prec))
            g.set_stream(stream.cuda_stream)
            g.kh_init(**cfg.kh_kwargs())
            g.upload()
            runs[prec] = g
        # step time of each form (after a few warm-up steps on a copy of the state)
        times = {}
        for prec, g in runs.items():
            g.step(3)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            g.step(10)
            e1.record(stream)
            torch.cuda.synchronize()
            times[prec] = e0.elapsed_time(e1) / 10
            g.kh_init(**cfg.kh_kwargs())
            g.upload()
        errs, done, breakdown = {}, 0, None
        from cueva import CuevaError
        for cp in checkpoints:
            try:
                for g in runs.values():
                    g.step(cp - done)
                    g.download()
            except CuevaError as e:
                breakdown = {"before_step": cp, "error": str(e)}
                break
            done = cp
            ref = {n: runs[0].interior(n).copy() for n in PRIM_NAMES}
            errs[str(cp)] = {n: rel_l1_field(n, runs[1].interior(n), ref[n], ref) for n in PRIM_NAMES}
            errs[str(cp) + "_vector"] = vector_rel_l1(runs[1], ref)
        out["variants"][label] = {"ms_per_step_fp64": times[0], "ms_per_step_mixed": times[1],
                                  "zone_updates_per_s_fp64": cfg.nx * cfg.ny / (times[0] * 1e-3),
                                  "zone_updates_per_s_mixed": cfg.nx * cfg.ny / (times[1] * 1e-3),
                                  "rel_l1_mixed_vs_fp64": errs, "breakdown": breakdown}
        for g in runs.values():
            g.close()
    print(json.dumps(out), flush=True)
    return 0


def run_mixed_learned(args, cfg, stream, g, device, world, pg):
    """FP32 reconstruction + Riemann with the learned con2prim seed (c2p = 2)
    over the same warm-up + timed steps from the same initial state as the
    FP64 run; its throughput and its per-variable error against that run."""
    import torch
    from cueva import Cueva
    from cueva.learned import LearnedSeed, learned_stats
    from cueva.metrics import rel_l1_field
    from cueva.train_seed import DEFAULT
    if not os.path.exists(DEFAULT):
        return {"unavailable": "no trained seed network: run python -m cueva.train_seed"}
    g.download()
    ref = {n: g.interior(n).copy() for n in PRIM_NAMES}
    net = LearnedSeed(device=device)
    net.load(DEFAULT)
    # one step from the initial state: mixed + learned, mixed + Cardano and FP64
    one = {}
    for prec, c2p in ((1, 2), (1, 1), (0, 1)):
        o = Cueva(device=device, pinned=False, **dict(cfg.solver_kwargs(), precision=prec, c2p=c2p))
        o.set_stream(stream.cuda_stream)
        o.kh_init(**cfg.kh_kwargs())
        o.upload()
        if c2p == 2:
            net.attach(o)
        o.step(1)
        o.download()
        one[(prec, c2p)] = {n: o.interior(n).copy() for n in PRIM_NAMES}
        o.close()
    one_err = {n: rel_l1_field(n, one[(1, 2)][n], one[(0, 1)][n], one[(0, 1)]) for n in PRIM_NAMES}
    # the same with v, E, B components measured against their vector's L1 norm
    one_vec = dict(one_err, **vector_rel_l1(one[(1, 2)], one[(0, 1)]))
    one_c2p = {n: rel_l1_field(n, one[(1, 2)][n], one[(1, 1)][n], one[(1, 1)]) for n in PRIM_NAMES}
    # error trajectory: plain FP64 and mixed + learned stepped side by side
    # from the initial state over the bench's step count; the largest
    # per-variable error (v, E, B components against their vector's L1
    # norm) after every step, and the step count up to which it stays <= 1e-6
    nsteps = max(args.warmup, 3) + args.steps
    traj = []
    runs = []
    for prec, c2p in ((0, 1), (1, 2)):
        o = Cueva(device=device, pinned=False, **dict(cfg.solver_kwargs(), precision=prec, c2p=c2p))
        o.set_stream(stream.cuda_stream)
        o.kh_init(**cfg.kh_kwargs())
        o.upload()
        if c2p == 2:
            net.attach(o)
        runs.append(o)
    for n in range(1, nsteps + 1):
        for o in runs:
            o.step(1)
            o.download()
        rf = {k: runs[0].interior(k) for k in PRIM_NAMES}
        e = dict({k: rel_l1_field(k, runs[1].interior(k), rf[k], rf) for k in PRIM_NAMES},
                 **vector_rel_l1(runs[1], rf))
        traj.append(max(e.values()))
    for o in runs:
        o.close()
    within = 0
    for n, e in enumerate(traj, 1):
        if e > 1e-6:
            break
        within = n
    m = Cueva(device=device, pinned=False, **dict(cfg.solver_kwargs(), precision=1, c2p=2))
    m.set_stream(stream.cuda_stream)
    m.kh_init(**cfg.kh_kwargs())
    m.upload()
    net.attach(m)
    m.step(max(args.warmup, 3))
    m.sync()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    m.step(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), pg)
    m.download()
    # the same mixed precision with the reference's Cardano recovery in the
    # last stage's update instead of the learned kernel, same steps
    mc = Cueva(device=device, pinned=False, **dict(cfg.solver_kwargs(), precision=1, c2p=1))
    mc.set_stream(stream.cuda_stream)
    mc.kh_init(**cfg.kh_kwargs())
    mc.upload()
    mc.step(max(args.warmup, 3))
    mc.sync()
    torch.cuda.synchronize()
    e0.record(stream)
    mc.step(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_card = max_over_ranks(e0.elapsed_time(e1), pg)
    mc.close()
    errs = {n: rel_l1_field(n, m.interior(n), ref[n], ref) for n in PRIM_NAMES}
    errs_vec = dict(errs, **vector_rel_l1(m, ref))
    its, pts, fails = learned_stats(m)
    prof_ms, prof_n = m.profile_steps(args.profile_steps) if args.profile_steps > 0 else ([0.0] * 3, [0] * 3)
    m.close()
    net.close()
    nprof = max(args.profile_steps, 1)
    return {"value": aggregate_rate(world, cfg.nx * cfg.ny, args.steps, ms), "unit": UNIT, "ms_per_step": ms / args.steps,
            "dtype": "f32 reconstruction + Riemann (psi, phi, E, B fluxes f64), f64 update / implicit E / con2prim",
            "con2prim": "network seed on the tcgen05 tensor cores (k_c2p_step), Newton in FP64, Cardano fall-back",
            "kernel_ms_per_step": dict({n: v[2] / nprof for n, v in stage_kernels(cfg, 4, prof_ms, prof_n).items()},
                                       k_c2p_step=prof_ms[2] / nprof),
            "rel_l1_learned_vs_cardano_one_step": one_c2p,
            "max_rel_l1_learned_vs_cardano_one_step": max(one_c2p.values()),
            "rel_l1_vs_fp64_one_step": one_err, "max_rel_l1_vs_fp64_one_step": max(one_err.values()),
            "rel_l1_vs_fp64_one_step_vector_norm": one_vec,
            "max_rel_l1_vs_fp64_one_step_vector_norm": max(one_vec.values()),
            "error_vs_fp64_after_steps": max(args.warmup, 3) + args.steps,
            "rel_l1_vs_fp64": errs, "max_rel_l1_vs_fp64": max(errs.values()),
            "rel_l1_vs_fp64_vector_norm": errs_vec, "max_rel_l1_vs_fp64_vector_norm": max(errs_vec.values()),
            "max_rel_l1_vs_fp64_vector_norm_by_step": traj, "steps_within_1e-6": within,
            "newton_iterations_per_point": its / max(pts, 1), "cardano_fallbacks": fails,
            "mixed_cardano": {"value": aggregate_rate(world, cfg.nx * cfg.ny, args.steps, ms_card),
                              "ms_per_step": ms_card / args.steps,
                              "note": "mixed precision with the reference's Cardano con2prim in the last "
                                      "stage's update, same steps"},
            "speedup_learned_vs_cardano": ms_card / ms}


ENS_METRIC = "ensemble zone-updates/s: 64 KH instances batched (mixed + learned C2P) vs sequential plain FP64"


def run_ensemble(args, quiet=False):
    """The batched-ensemble workload: 64 KH instances (seed 2024) in one
    CUDA-graph step per ensemble step, launch shape picked by the autotuner;
    mixed precision + learned con2prim seed, against the same 64 instances
    run one after another in plain FP64 (and the batched FP64 form)."""
    import torch
    from cueva import Cueva
    from cueva.ensemble import Ensemble, kh_ensemble
    from cueva.learned import LearnedSeed
    from cueva.metrics import rel_l1_field
    from cueva.train_seed import DEFAULT
    insts = kh_ensemble(args.ens_n, seed=2024)
    common = dict(order=4, flux_solver=7, rec_mp=0, intsum_reset=1)
    zones = sum(i.nx * i.ny for i in insts)
    warm, K = max(args.warmup, 3), args.steps
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)

    def timed_ensemble(precision, c2p):
        ens = Ensemble([i.solver_kwargs(**common, precision=precision, c2p=c2p) for i in insts])
        ens.set_stream(stream.cuda_stream)
        net = None
        if c2p == 2:
            net = LearnedSeed()
            net.load(DEFAULT)
            ens.attach(net)
        for k, i in enumerate(insts):
            ens.kh_init(k, **i.kh_kwargs())
        tune = ens.autotune()
        ens.step(warm)
        ens.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ens.step(K)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        ens.sync()
        return ens, net, ms, tune

    mixed, net, ms_mixed, tune_mixed = timed_ensemble(1, 2)
    its, pts, fails = mixed.learned_stats()
    fp64, _, ms_fp64, tune_fp64 = timed_ensemble(0, 1)
    errs = []
    for k in range(len(insts)):
        ref = fp64.get_prims(k)
        got = mixed.get_prims(k)
        errs.append(max(rel_l1_field(n, got[n], ref[n], ref) for n in ("rho", "p", "vx", "vy", "By", "Ez")))
    mixed.close()
    fp64.close()
    if net is not None:
        net.close()
    # the same instances one after another, plain FP64, one context each
    ms_seq = 0.0
    for i in insts:
        g = Cueva(**i.solver_kwargs(**common))
        g.set_stream(stream.cuda_stream)
        g.kh_init(**i.kh_kwargs())
        g.upload()
        g.step(warm)
        g.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        g.step(K)
        e1.record(stream)
        torch.cuda.synchronize()
        ms_seq += e0.elapsed_time(e1)
        g.close()

    def rate(ms):
        return zones * K / (ms * 1e-3)

    sizes = {}
    for i in insts:
        sizes[f"{i.nx}x{i.ny}"] = sizes.get(f"{i.nx}x{i.ny}", 0) + 1
    line = {"metric": ENS_METRIC, "value": rate(ms_mixed), "unit": UNIT, "n_gpus": 1, "steps": K, "warmup": warm,
            "ms_per_step": ms_mixed / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 reconstruction + Riemann (psi, phi, E, B fluxes f64), f64 update / implicit E / con2prim (learned seed)",
            "data": "synthetic KH ensemble (seed 2024)",
            "config": {"workload": f"kh-ensemble-{len(insts)}", "instances": len(insts), "zones": zones,
                       "grids": sizes, "solver": "MP5+HLLC", "imex": "SSP3(4,3,3), stage sums reset per stage"},
            "autotune": {"rows": tune_mixed[0], "ctas_per_sm": tune_mixed[1], "ms_per_step": tune_mixed[2]},
            "batched_fp64": {"value": rate(ms_fp64), "ms_per_step": ms_fp64 / K,
                             "autotune": {"rows": tune_fp64[0], "ctas_per_sm": tune_fp64[1]}},
            "sequential_fp64": {"value": rate(ms_seq), "ms_per_step": ms_seq / K},
            "speedup_vs_sequential_fp64": ms_seq / ms_mixed,
            "rel_l1_mixed_vs_fp64": {"median": float(sorted(errs)[len(errs) // 2]), "max": float(max(errs)),
                                     "after_steps": warm + K},
            "learned": {"newton_iterations_per_point": its / max(pts, 1), "cardano_fallbacks": fails}}
    if quiet:
        return line
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", type=int, default=0, help="0 FP64, 1 mixed")
    ap.add_argument("--c2p", type=int, default=1, help="1 Cardano (reference), 0 NR, 2 learned seed + Newton")
    ap.add_argument("--stage-kernel", type=int, default=None,
                    help="1 one fused kernel per RK stage, 0 the y-face + x-face/update kernels (default: fused)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--profile-steps", type=int, default=3)
    ap.add_argument("--grid", default=None, help="NXxNY override of the workload grid (profiling a small case)")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed + learned-seed measurement")
    ap.add_argument("--mixed-study", action="store_true",
                    help="per-variable error and speed of mixed precision vs FP64 (2048x4096, MP7/MP9)")
    ap.add_argument("--study-steps", default="1,100,150,1000")
    ap.add_argument("--ensemble", action="store_true", help="the 64-instance batched KH ensemble workload")
    ap.add_argument("--ens-n", type=int, default=64)
    ap.add_argument("--no-ensemble", action="store_true", help="skip the ensemble measurement of the default run")
    args = ap.parse_args()

    from cueva.configs import TARGET
    cfg = TARGET
    if args.grid:
        import dataclasses
        nx, ny = (int(v) for v in args.grid.lower().split("x"))
        cfg = dataclasses.replace(TARGET, nx=nx, ny=ny, name=TARGET.name.replace("2048x4096", f"{nx}x{ny}"))
    if args.impl == "reference":
        return run_reference(args, cfg)
    if args.mixed_study:
        return mixed_study(args)
    if args.ensemble:
        return run_ensemble(args)

    import numpy as np
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist
    from cueva import Cueva

    g = Cueva(device=local, pinned=True, **dict(cfg.solver_kwargs(), precision=args.precision, c2p=args.c2p))
    if args.stage_kernel is not None:
        g.set_stage_kernel(args.stage_kernel)
    if args.c2p == 2:
        from cueva.learned import LearnedSeed
        from cueva.train_seed import DEFAULT
        seed_net = LearnedSeed(device=local)
        seed_net.load(DEFAULT)
        seed_net.attach(g)
    # a dedicated (non-default) stream shared by the library and the CUDA events
    stream = torch.cuda.Stream(device=local)
    torch.cuda.set_stream(stream)
    g.set_stream(stream.cuda_stream)
    g.kh_init(**cfg.kh_kwargs())
    g.upload()
    s = g.lmax

    def barrier():
        torch.cuda.synchronize()
        if pg is not None:
            pg.barrier()
            torch.cuda.synchronize()

    for _ in range(max(args.warmup, 3)):
        g.step(1)
    g.sync()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        g.step(args.steps)
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    g.sync()                                    # raises on a reference STOP condition
    ms_max = max_over_ranks(ms, pg)
    zones = cfg.nx * cfg.ny
    value = aggregate_rate(world, zones, args.steps, ms_max)
    ms_per_step = ms_max / args.steps

    # the mixed-precision + learned-seed form on the same workload and steps
    mixed = None if args.no_mixed else run_mixed_learned(args, cfg, stream, g, local, world, pg)

    # end to end through the C-ABI with host buffers: per step the 14 prim
    # fields go up from pinned host arrays, one time step runs, and they come
    # back down.  The asynchronous readback lets field f of step k go back up
    # while field f+1 still comes down (the two directions use separate copy
    # engines); the synchronous loop is measured beside it.
    def e2e_loop(async_readback):
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.e2e_steps):
            g.upload()
            g.step(1)
            if async_readback:
                g.download_async()
            else:
                g.download()
        g.sync()                                # the last readback is complete
        e1.record(stream)
        torch.cuda.synchronize()
        ms_ = max_over_ranks(e0.elapsed_time(e1), pg)
        return aggregate_rate(world, zones, args.e2e_steps, ms_)

    e2e_sync = e2e_loop(False)
    e2e_async = e2e_loop(True)
    field_bytes = 14 * zones_pts(cfg) * 8
    e2e = {"value": e2e_async, "unit": UNIT,
           "h2d_bytes_per_step": field_bytes, "d2h_bytes_per_step": field_bytes,
           "synchronous_download_value": e2e_sync,
           "note": "per step: upload of the 14 prim fields from pinned host arrays, one time step, "
                   "download_async (field-ordered readback overlapping the next upload); "
                   "the last readback is synchronised inside the timed region"}

    # per-kernel device time: a few steps launched kernel by kernel with
    # events between the launches on the library's stream
    peak, peak_kind = measured_peaks()
    kms, kcnt = g.profile_steps(args.profile_steps)
    g.sync()
    kernels = {}
    for name, (units, bpu, ms_sum, cnt) in stage_kernels(cfg, s, kms, kcnt).items():
        avg = ms_sum / max(cnt, 1)
        kernels[name] = {"avg_ms": avg, "launches": cnt, "share": ms_sum / max(sum(kms), 1e-30), "units": units,
                         "alg_bytes_per_unit": bpu, "alg_bytes_per_launch": bpu * units,
                         "gbs": bpu * units / (avg * 1e-3) / 1e9 if avg > 0 else None}
    top = max(kernels, key=lambda n: kernels[n]["avg_ms"] * kernels[n]["launches"])
    achieved = kernels[top]["gbs"]
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "kernel_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            tr = json.load(f)
        per_unit = tr.get("kernels", {}).get(top, {}).get("dram_bytes_per_unit")
        if per_unit is not None:
            traffic = per_unit * kernels[top]["units"]
    clocks = clk.summary()
    roof_fp64 = fp64_roofline(kernels, top, clocks.get("sm_mhz"))
    step_bytes = alg_bytes_per_zone(s) * zones_pts(cfg)
    launches_per_step = sum(kcnt) / max(args.profile_steps, 1)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if args.precision == 0 else "f64+f32",
            "data": f"synthetic KH initial data ({cfg.nx} x {cfg.ny} shear layer, reference orientation)",
            "config": {"workload": cfg.name, "nx": cfg.nx, "ny": cfg.ny, "points": zones_pts(cfg), "rk_stages": s,
                       "solver": "MP5+HLLC", "imex": "SSP3(4,3,3), stage sums reset per stage",
                       "sigma": cfg.sigma,
                       "precision": "fp64" if args.precision == 0 else "mixed",
                       "l2": f"working set {g.device_bytes() / 1e9:.1f} GB on the device >> 126 MB L2 "
                             "(no flush needed)",
                       "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_kind": peak_kind,
                         "kernel": top, "kernels": kernels,
                         "whole_step_gbs": step_bytes / (ms_per_step * 1e-3) / 1e9,
                         "whole_step_frac": step_bytes / (ms_per_step * 1e-3) / 1e9 / peak,
                         "note": f"{top}: {kernels[top]['alg_bytes_per_unit']:.0f} algorithmic B per unit x "
                                 f"{kernels[top]['units']} units per launch / avg launch "
                                 f"{kernels[top]['avg_ms']:.3f} ms; whole step: B_alg(s) = "
                                 f"{alg_bytes_per_zone(s):.0f} B per point over the timed ms per step; "
                                 "traffic: DRAM bytes per unit of an ncu capture (profiles/kernel_traffic.json) "
                                 "times the units of a launch"},
            "roofline_fp64": roof_fp64,
            "clocks": clocks, "e2e": e2e, "gpu_launches": int(round(launches_per_step * args.steps)),
            "mixed_learned": mixed}
    if rank == 0 and not args.no_ensemble:
        # the 64-instance ensemble workload (its own line with --ensemble)
        try:
            line["ensemble"] = run_ensemble(args, quiet=True)
        except Exception as e:   # reported, not fatal: the headline above stands on its own
            line["ensemble"] = {"unavailable": f"{type(e).__name__}: {e}"}
        torch.cuda.set_stream(stream)
    if rank == 0 and not args.no_cpu_baseline:
        r, cores, sample = cpu_port_rate(cfg)
        line["cpu_baseline"] = {"value": r, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}
    if rank == 0:
        print(json.dumps(line), flush=True)
    g.close()
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def zones_pts(cfg):
    return (cfg.imax + 1) * (cfg.jmax + 1)


if __name__ == "__main__":
    sys.exit(main())
