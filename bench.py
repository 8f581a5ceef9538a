#!/usr/bin/env python
"""Benchmark of LOQUAT's per-step SPH path on B200: particle-steps/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (default): 3D cylinder collapse, R = 0.2 m, H = 0.4 m,
dr = 2.949 mm (about 1.96 M soil particles) on a 3-layer Adami floor,
Drucker-Prager phi = 30 deg, E = 5 MPa, nu = 0.3, rho = 2000 kg/m^3,
Wendland C2 with h = 1.3 dr, mixed-precision form (the plain FP32 form is
timed in the same run).  Seeded synthetic input.
One step = predictor + corrector stages (search, gather, Adami,
interaction, integration) plus the Shepard pass every 30 steps.

`value` is material particle-steps/s of the whole job with the state
resident in HBM (device time, CUDA events on the simulation's stream, max
over ranks).  `e2e` is the same metric through the C ABI from pinned host
buffers: state upload, every step followed by a device->host read of the
16-byte health word, and the final state download, all inside the timed
region.  Under torchrun every rank runs an independent replica (weak
scaling, no collective in the data path).

The default run adds three legs to the line: `amortized` (a 250-step
window of the same run, carrying the neighbour-list rebuilds at their
natural rate), `dropin` (the reference's step sequence through the drop-in
entry points on the same workload) and `ensemble` (config 4: 256 batched
scenarios in both precision forms against the same scenarios run one
after another, each side autotuned).

`--impl reference` times the CPU FP64 OpenMP restatement of the reference's
algorithm (the reference has no CPU implementation of its own and its GPU
build cannot be assembled: two of its libraries are not distributed) on the
same workload, with every host thread and then on one thread; it derives
the case's Parameters with the oracle and loads no library of the product.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

BYTES_INTERACTION_PER_PARTICLE = 112   # 56 B read (pos, velrhop, str) + 56 B written (accad, spin, acestn)
# FP32 operations per list entry of the pair kernel (k_interaction_rec's
# pair body with artificial viscosity on and artificial stress off, an FMA
# counted as 2, MUFU sqrt / reciprocal as 1): distance and kernel gradient
# 18, density rate 6, momentum 21, viscosity 19, velocity difference and
# gradient 24, momentum sums 3, neighbour volume 2 (93); the compensated sums
# of the mixed form add 12.
FLOPS_PER_ENTRY = {"plain": 93, "mixed": 105}
FP32_PEAK_NOMINAL = 148 * 128 * 2 * 1.965e9 / 1e12   # TFLOP/s: SMs x FP32 lanes x FMA x max SM clock


def parse_args(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=250)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=["cylinder", "column", "ensemble", "slope", "inclined"], default="cylinder",
                    help="slope / inclined: the von Wolffersdorff workloads (2.85 M soil at dr 5 mm; 16.0 M at "
                         "dr 2.5 mm)")
    ap.add_argument("--scenarios", type=int, default=256, help="ensemble size (--config ensemble)")
    ap.add_argument("--dr", type=float, default=None, help="override the particle spacing")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--form", choices=["plain", "mixed"], default="mixed",
                    help="plain FP32, or mixed precision (FP64 integrator accumulation and stress update, "
                         "compensated interaction sums)")
    ap.add_argument("--profile-steps", type=int, default=10)
    ap.add_argument("--start-step", type=int, default=None,
                    help="untimed steps run first so the timed window sits mid-run of the 5000-step collapse "
                         "(the particles move and the neighbour lists are rebuilt at a representative rate); "
                         "default 2500, 200 for the von Wolffersdorff workloads")
    ap.add_argument("--no-compare", action="store_true", help="skip timing the other precision form")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default pair-kernel shape and list skin instead of lq_sim_autotune's choice")
    ap.add_argument("--tune-steps", type=int, default=40, help="timed steps per autotuner trial")
    ap.add_argument("--pair-shape", type=int, default=None,
                    help="fix the pair kernel's launch shape (lq_sim_set_pair_shape, 0-10) instead of autotuning")
    ap.add_argument("--skin", type=float, default=None,
                    help="with --pair-shape: the list skin / h (lq_sim_set_skin; default 0.05)")
    ap.add_argument("--wide", type=float, default=None,
                    help="with --pair-shape: two-level lists' wide cut-off beyond 2h, / h (lq_sim_set_wide_skin)")
    ap.add_argument("--no-dropin", action="store_true",
                    help="skip timing the reference's step sequence through the drop-in entry points")
    ap.add_argument("--no-ensemble", action="store_true",
                    help="skip the config-4 ensemble leg of the default run")
    ap.add_argument("--amortized-steps", type=int, default=250,
                    help="length of the second, longer timed window that carries the neighbour-list rebuilds at "
                         "their natural rate (0 to skip)")
    ap.add_argument("--eager", action="store_true",
                    help="launch kernels one by one instead of replaying the step graph (for ncu, which cannot "
                         "profile kernels inside graphs with conditional nodes)")
    a = ap.parse_args(argv)
    if a.start_step is None:
        a.start_step = 200 if a.config in ("slope", "inclined") else 2500
    return a


def make_case(args, rank=0):
    from loquat_b200 import cases

    if args.config == "cylinder":
        kw = {} if args.dr is None else {"dr": args.dr}
        return cases.cylinder_collapse(seed=1 + rank, **kw)
    kw = {} if args.dr is None else {"dr": args.dr}
    if args.config == "slope":
        return cases.slope_failure(seed=1 + rank, **kw)
    if args.config == "inclined":
        return cases.inclined_block(seed=1 + rank, **kw)
    return cases.column_collapse(seed=1 + rank, **kw)


def cpu_sample_case(args):
    """Bounded CPU sample of the workload: the same material, spacing and
    smoothing length on a cylinder scaled down to about 100 k soil particles."""
    from loquat_b200 import cases

    if args.config == "cylinder":
        s = (1.0e5 / 1.96e6) ** (1.0 / 3.0)
        return cases.cylinder_collapse(radius=0.2 * s, height=0.4 * s, seed=1), "cylinder R=%.4f m H=%.4f m" % (
            0.2 * s, 0.4 * s)
    if args.config in ("slope", "inclined"):
        s = (1.0e5 / 2.856e6) ** (1.0 / 3.0)
        return cases.slope_failure(dr=0.005 / s, seed=1), "slope failure at dr=%.2f mm (~100 k soil)" % (5.0 / s)
    return cases.column_collapse(seed=1), "column collapse 50k"


def workload_config(args, par):
    """The line's `config`: the workload and its sizes, the same in both arms."""
    return {"workload": workload_name(args), "np": par.np, "npm": par.npm, "npb": par.npb, "ncell": par.ncell}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_from_profiles(workload: str, form: str):
    """ncu figures of the pair kernel for this workload and form from the
    committed summary (profiles/interaction_traffic.json), if any:
    {"traffic": DRAM bytes per launch, ...}."""
    f = ROOT / "profiles" / "interaction_traffic.json"
    if not f.exists():
        return None
    try:
        d = json.loads(f.read_text())
        return d.get(f"{workload} [{form}]")
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str | None):
        self.proc = None
        self.path = None
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
            if gpu_id:
                cmd += ["-i", gpu_id]
            self.proc = subprocess.Popen(cmd, stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def gpu_uuid(torch, dev):
    try:
        return "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        return None


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_cpu_baseline(args, steps=5, warmup=1):
    """The FP64 oracle on all host threads on the bounded sample."""
    import oracle

    case, desc = cpu_sample_case(args)
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    sim = oracle.OracleSim(case.par, *case.arrays())
    if "hypoplastic" in case.meta:
        sim.set_vw(case.meta["hypoplastic"])
    sim.step(warmup)
    t0 = time.perf_counter()
    sim.step(steps)
    dt = time.perf_counter() - t0
    sim.close()
    value = case.par.npm * steps / dt
    return {"value": value, "unit": "particle-steps/s", "cores": threads, "kind": "port",
            "sample": f"{desc} at dr={case.meta['dr'] * 1e3:.3f} mm ({case.par.npm} soil + {case.par.npb} boundary "
                      f"particles), {warmup} warm-up + {steps} timed steps, FP64"}, dt


# the CPU arm times at most this many particle-steps per leg (about a minute
# of FP64 work on 16 host threads); larger workloads run fewer timed steps
REFERENCE_BUDGET_PARTICLE_STEPS = 1.2e8


def bench_reference(args):
    """The reference's algorithm on the host: the FP64 OpenMP restatement
    (oracle/) of reference src/loquat.cu:322-409 on the same workload as
    the GPU arm, with every host thread, then the same state stepped on one
    thread.  The case's Parameters are derived by the oracle, so this arm
    loads no library of the product."""
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    if args.config == "ensemble":
        print(json.dumps({"impl": "reference", "unavailable": "the CPU arm times the single-domain workloads; the "
                                                              "ensemble's 30 M particles exceed its budget"}))
        return 0
    import oracle
    from loquat_b200 import cases

    cases.use_parameter_initializer(oracle.initialize_parameters)
    case = make_case(args)
    par = case.par
    threads = os.cpu_count() or 1
    steps = max(1, min(args.steps, int(REFERENCE_BUDGET_PARTICLE_STEPS // max(par.np, 1))))
    oracle.set_threads(threads)
    sim = oracle.OracleSim(par, *case.arrays())
    if "hypoplastic" in case.meta:
        sim.set_vw(case.meta["hypoplastic"])
    sim.step(min(args.warmup, 2))
    t0 = time.perf_counter()
    sim.step(steps)
    dt = time.perf_counter() - t0
    value = par.npm * steps / dt
    # the same state, one host thread, one step (reference-free single-core figure)
    oracle.set_threads(1)
    t1 = time.perf_counter()
    sim.step(1)
    dt1 = time.perf_counter() - t1
    sim.close()
    single = par.npm / dt1
    sample = (f"the full workload ({par.npm} soil + {par.npb} boundary particles), {steps} timed steps after "
              f"{min(args.warmup, 2)} warm-up steps")
    out = {
        "impl": "reference",
        "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": args.gpus,
        "steps": steps, "warmup": min(args.warmup, 2), "ms_per_step": 1e3 * dt / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args, par),
        "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": threads, "kind": "port",
                         "sample": sample + ", FP64 OpenMP restatement of the reference algorithm"},
        "single_thread": {"value": single, "unit": "particle-steps/s", "cores": 1,
                          "sample": "one further step of the same state on one host thread"},
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))
    return 0


def workload_name(args):
    if args.config == "cylinder":
        return "cylinder collapse R=0.2 m H=0.4 m dr=%.3f mm h=1.3dr DP phi=30" % (1e3 * (args.dr or 0.002949))
    if args.config == "slope":
        return ("von Wolffersdorff slope failure 2.0x0.6x0.35 m at 45 deg dr=%.1f mm h=1.2dr e0=0.70 "
                "(FP64 sub-stepping, tol 1e-4)" % (1e3 * (args.dr or 0.005)))
    if args.config == "inclined":
        return ("von Wolffersdorff 1.0x1.0x0.25 m block on a 30 deg plane dr=%.1f mm h=1.2dr e0=0.65 "
                "(FP64 sub-stepping, tol 1e-4)" % (1e3 * (args.dr or 0.0025)))
    return "column collapse 0.2x0.1x0.02 m dr=2 mm h=1.2dr DP phi=19.8"


def dropin_measurement(args, case, torch, dist):
    """The reference's step sequence (src/loquat.cu:322-409: a search and
    re-sort before each stage, Adami, ParticleInteraction, Predictor /
    Corrector, Shepard every N steps) through the drop-in entry points on
    the same workload, as a caller of the reference's headers runs it;
    CUDA events on its stream, max over ranks."""
    from loquat_b200 import dropin, replicas

    stream = torch.cuda.Stream()
    seq = dropin.ReferenceStep(case.par, *case.arrays(), stream=stream)
    seq.step(args.warmup)
    stream.synchronize()
    if dist:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    seq.step(args.steps)
    e1.record(stream)
    stream.synchronize()
    ms = replicas.max_over_ranks(e0.elapsed_time(e1), device="cuda")
    # one ParticleInteraction call on its own (cell starts, tile order,
    # list build in the caller's grid, pack, pair kernel)
    from loquat_b200 import particle_interaction

    beg, end = seq._cells()
    calls = 5
    i0, i1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    i0.record(stream)
    for _ in range(calls):
        particle_interaction(seq.par, seq.par_dev, *seq.state, *seq.rates, beg, end, stream=seq._s)
    i1.record(stream)
    stream.synchronize()
    call_ms = replicas.max_over_ranks(i0.elapsed_time(i1) / calls, device="cuda")
    seq.close()
    world = dist.get_world_size() if dist else 1
    return {"value": case.par.npm * args.steps * world / (ms / 1e3), "unit": "particle-steps/s",
            "ms_per_step": ms / args.steps, "steps": args.steps, "interaction_ms_per_call": call_ms,
            "form": "plain FP32, the reference's call sequence through lq_grid_*, lq_adami_boundary, "
                    "lq_particle_interaction, lq_predictor / lq_corrector, lq_stress_regularization"}


def bench_ours(args):
    import torch

    world, rank, local = dist_setup()
    if not torch.cuda.is_available():
        print(json.dumps({"error": "no CUDA device"}))
        return 1
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    import loquat_b200 as lq

    case = make_case(args, rank)
    par = case.par
    npm, np_ = par.npm, par.np
    sim = lq.Simulation(par, *case.arrays(), graph=not args.eager, mixed=args.form == "mixed")
    if "hypoplastic" in case.meta:
        sim.set_hypoplastic(case.meta["hypoplastic"])
    ext = torch.cuda.ExternalStream(sim.stream())
    plain, with_shep = sim.launches_per_step()

    tuned = None
    if args.pair_shape is not None:
        # a fixed shape and lists apply to the whole run (profiling runs)
        sim.set_pair_shape(args.pair_shape)
        skin = 0.05 if args.skin is None else args.skin
        sim.set_skin(skin)
        if args.wide is not None:
            sim.set_wide_skin(args.wide)
        tuned = {"pair_shape": args.pair_shape, "skin_over_h": skin, "wide_over_h": sim.wide_skin(),
                 "steps_per_trial": 0}
    if args.start_step > 0:
        sim.step(args.start_step)
    if args.pair_shape is None and not args.no_autotune:
        # the project's autotuner: pair-kernel launch shape and list skin by
        # timing, the state left as it was (outside the timed region)
        shape, skin = sim.autotune(args.tune_steps)
        tuned = {"pair_shape": shape, "skin_over_h": skin, "wide_over_h": sim.wide_skin(),
                 "steps_per_trial": args.tune_steps}
    sim.step(args.warmup)
    sim.synchronize()
    rb0, rn0 = sim.rebuilds(), sim.renewals()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    s0, _ = sim.clock()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(gpu_uuid(torch, local)) if rank == 0 else None
    start.record(ext)
    sim.step(args.steps)
    end.record(ext)
    sim.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop() if clocks else None
    s1, _ = sim.clock()
    from loquat_b200 import replicas
    ms = replicas.max_over_ranks(start.elapsed_time(end), device="cuda")
    shep_steps = sum(1 for s in range(s0, s1) if par.stress_shepard_filter and s % par.stress_shepard_filter == 0
                     and s != 0)
    rebuilds, renewals = sim.rebuilds() - rb0, sim.renewals() - rn0
    launches = ((s1 - s0) * plain + shep_steps * (with_shep - plain) + rebuilds * sim.rebuild_launches()
                + renewals * sim.renewal_launches())
    value = npm * args.steps * world / (ms / 1e3)
    health = sim.health()

    # a longer window of the same run: its rebuilds come at their natural
    # rate, so its time per step carries their amortised cost
    amortized = None
    if args.amortized_steps > 0:
        rb_a, rn_a = sim.rebuilds(), sim.renewals()
        sim.synchronize()
        if dist:
            dist.barrier()
        aext = torch.cuda.ExternalStream(sim.stream())
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(aext)
        sim.step(args.amortized_steps)
        a1.record(aext)
        sim.synchronize()
        ams = replicas.max_over_ranks(a0.elapsed_time(a1), device="cuda")
        amortized = {"form": args.form, "value": npm * args.amortized_steps * world / (ams / 1e3),
                     "ms_per_step": ams / args.amortized_steps, "steps": args.amortized_steps,
                     "neighbour_list_rebuilds": sim.rebuilds() - rb_a,
                     "neighbour_list_renewals": sim.renewals() - rn_a}

    # live per-phase device times (eager launches, CUDA events on the same stream)
    prof = sim.profile(args.profile_steps) if args.profile_steps > 0 else {}
    inter_ms, inter_n = prof.get("interaction", (0.0, 0))
    t_int = inter_ms / max(inter_n, 1) / 1e3
    peak, peak_kind = measured_peaks()
    achieved_gbs = BYTES_INTERACTION_PER_PARTICLE * npm / t_int / 1e9 if t_int > 0 else None
    workload = workload_name(args)
    ncu = traffic_from_profiles(workload, args.form)
    traffic = ncu.get("traffic") if ncu else None
    entries, _ = sim.neighbor_entries()
    flops = FLOPS_PER_ENTRY[args.form] * entries
    achieved_tf = flops / t_int / 1e12 if t_int > 0 else None

    e2e = None
    if not args.no_e2e:
        host = [torch.empty(a.shape, dtype=torch.float32, pin_memory=True).numpy() for a in case.arrays()]
        for h, a in zip(host, case.arrays()):
            h[...] = a
        out = [torch.empty(a.shape, dtype=torch.float32, pin_memory=True).numpy() for a in case.arrays()]
        sim.synchronize()
        if dist:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        sim.upload(*host)
        for _ in range(args.steps):
            sim.step(1)
            sim.health()             # device -> host read of the step's result
        sim.download(out)
        e1.record(ext)
        sim.synchronize()
        ems = replicas.max_over_ranks(e0.elapsed_time(e1), device="cuda")
        state_bytes = sum(a.nbytes for a in host)
        e2e = {"value": npm * args.steps * world / (ems / 1e3), "unit": "particle-steps/s",
               "h2d_bytes_per_step": state_bytes / args.steps,
               "d2h_bytes_per_step": (state_bytes + 16 * args.steps) / args.steps}

    # the other precision form on the same workload and window, for comparison
    forms = {args.form: {"value": value, "ms_per_step": ms / args.steps}}
    if not args.no_compare:
        other = "plain" if args.form == "mixed" else "mixed"
        sim.close()
        osim = lq.Simulation(par, *case.arrays(), graph=not args.eager, mixed=other == "mixed")
        if "hypoplastic" in case.meta:
            osim.set_hypoplastic(case.meta["hypoplastic"])
        if args.start_step > 0:
            osim.step(args.start_step)
        other_tuned = tuned
        if args.pair_shape is None and not args.no_autotune:
            # each form tuned on its own: its best launch shape and skin
            shape, skin = osim.autotune(args.tune_steps)
            other_tuned = {"pair_shape": shape, "skin_over_h": skin, "wide_over_h": osim.wide_skin(),
                           "steps_per_trial": args.tune_steps}
        elif tuned:
            osim.set_pair_shape(tuned["pair_shape"])
            osim.set_skin(tuned["skin_over_h"])
            osim.set_wide_skin(tuned.get("wide_over_h", 0.0))
        osim.step(args.warmup)
        osim.synchronize()
        if dist:
            dist.barrier()
        oext = torch.cuda.ExternalStream(osim.stream())
        o0, o1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        o0.record(oext)
        osim.step(args.steps)
        o1.record(oext)
        osim.synchronize()
        oms = replicas.max_over_ranks(o0.elapsed_time(o1), device="cuda")
        forms[other] = {"value": npm * args.steps * world / (oms / 1e3), "ms_per_step": oms / args.steps,
                        "autotuned": other_tuned}
        sim = osim

    sim.close()
    sim = None

    dropin = None
    if not args.no_dropin and args.config in ("cylinder", "column"):
        dropin = dropin_measurement(args, case, torch, dist)

    ensemble = None
    if not args.no_ensemble and args.config == "cylinder":
        # a window long enough that list sorts and renewals come at their
        # natural rate (the line's own value keeps exactly --steps steps)
        ensemble = ensemble_measurement(args, torch, world, rank, local, dist,
                                        steps=max(args.steps, ENSEMBLE_KEY_STEPS))

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, _ = run_cpu_baseline(args)

    if rank == 0:
        line = {
            "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32" if args.form == "plain" else "f32+f64", "data": "synthetic",
            "config": workload_config(args, par),
            "run": {"autotuned": tuned,
                    "form": "%s, %s, Verlet lists" % (
                        "plain FP32" if args.form == "plain" else "mixed precision (FP64 integrator)",
                        "eager launches" if args.eager else "CUDA-graph step"),
                    "timed_window": "steps %d..%d of the run" % (s0, s1),
                    "l2": "state larger than L2 (3 x %.0f MB state buffers)" % (np_ * 96 / 1e6),
                    "parallelism": f"{world} independent replicas" if world > 1 else "single GPU"},
            "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": peak, "unit": "GB/s",
                         "frac": (achieved_gbs / peak) if achieved_gbs else None, "traffic": traffic,
                         "kernel": "k_interaction_rec", "peak_kind": peak_kind,
                         "bytes_per_launch": BYTES_INTERACTION_PER_PARTICLE * npm,
                         "ms_per_launch": t_int * 1e3,
                         "ncu": ncu},
            "roofline_fp32": {"achieved": achieved_tf, "peak": FP32_PEAK_NOMINAL, "unit": "TFLOP/s",
                              "frac": (achieved_tf / FP32_PEAK_NOMINAL) if achieved_tf else None,
                              "peak_kind": "nominal (no measured FP32 peak)",
                              "flops_per_launch": flops, "list_entries": entries,
                              "flops_per_entry": FLOPS_PER_ENTRY[args.form]},
            "phases_ms_per_step": {k: v[0] / max(args.profile_steps, 1) for k, v in prof.items()},
            "forms": forms,
            "gpu_launches": launches,
            "neighbour_list_rebuilds": rebuilds,
            "neighbour_list_renewals": renewals,
            "health": [int(x) for x in health],
            "clocks": clk,
            "e2e": e2e,
            "amortized": amortized,
            "dropin": dropin,
            "ensemble": ensemble,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def size_classes(counts, nclass=4):
    """Scenario indices grouped by particle count into nclass log-spaced
    classes (empty classes dropped)."""
    c = np.log(np.asarray(counts, np.float64))
    lo, hi = c.min(), c.max() + 1e-9
    cls = np.minimum(((c - lo) / max(hi - lo, 1e-9) * nclass).astype(int), nclass - 1)
    return [list(np.nonzero(cls == k)[0]) for k in range(nclass) if np.any(cls == k)]


# timed steps of the ensemble measurement carried by the default line, and
# steps of its per-phase profile
ENSEMBLE_KEY_STEPS = 100
ENSEMBLE_PROFILE_STEPS = 40


def ensemble_measurement(args, torch, world, rank, local, dist, sample_clocks=False, steps=None):
    """Batched ensemble of config 4 (one simulation holding every scenario,
    one graph launch per step) in both precision forms, against the same
    scenarios run one after another, each as its own plain simulation.  The
    batched forms are autotuned as a whole; the sequential runs are tuned by
    size class (one autotuner run on the median scenario of each of four
    log-spaced particle-count classes, its shape and skin applied to the
    class).  All timed with CUDA events on the simulations' streams after
    the same warm-up; max over ranks.  `steps` (default --steps) is the
    timed window of every run."""
    import loquat_b200 as lq
    from loquat_b200 import cases, replicas

    _, all_parts = cases.ensemble(n=args.scenarios, seed=4)
    shares = replicas.partition([p.par.npm for p in all_parts], world)
    parts = [all_parts[k] for k in shares[rank]]
    comb = cases.combine(parts)
    par = comb.par
    nsteps = steps or args.steps
    total_npm = sum(p.par.npm for p in all_parts)

    def timed(sim, steps):
        ext = torch.cuda.ExternalStream(sim.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        sim.synchronize()
        e0.record(ext)
        sim.step(steps)
        e1.record(ext)
        sim.synchronize()
        return e0.elapsed_time(e1)

    def batched(mixed):
        sim = lq.Simulation(par, *comb.arrays(), mixed=mixed, graph=not args.eager)
        sim.set_materials(comb.meta["materials"])
        sim.set_frames(comb.meta["frames"])
        sim.step(args.warmup)
        tuned = None
        if not args.no_autotune:
            shape, skin = sim.autotune(args.tune_steps)
            tuned = {"pair_shape": shape, "skin_over_h": skin, "wide_over_h": sim.wide_skin(),
                     "steps_per_trial": args.tune_steps}
        return sim, tuned

    forms, tuned_by_form, extra = {}, {}, {}
    for form in (args.form, "plain" if args.form == "mixed" else "mixed"):
        sim, tuned = batched(form == "mixed")
        rb0, rn0 = sim.rebuilds(), sim.renewals()
        sim.synchronize()
        if dist:
            dist.barrier()
        clocks = ClockSampler(gpu_uuid(torch, local)) if (sample_clocks and rank == 0 and not forms) else None
        ms = replicas.max_over_ranks(timed(sim, nsteps), device="cuda")
        if not forms:
            extra = {"clocks": clocks.stop() if clocks else None, "neighbour_list_rebuilds": sim.rebuilds() - rb0,
                     "neighbour_list_renewals": sim.renewals() - rn0,
                     "health": [int(x) for x in sim.health()], "gpu_launches_per_step": sim.launches_per_step()[0]}
            if args.profile_steps > 0:
                # per-phase device times of the same run (eager launches, CUDA
                # events; long enough to hold sorts and renewals at their rate)
                n = max(args.profile_steps, ENSEMBLE_PROFILE_STEPS)
                prof = sim.profile(n)
                extra["phases_ms_per_step"] = {k: v[0] / n for k, v in prof.items()}
                extra["phase_launches"] = {k: v[1] for k, v in prof.items()}
        sim.close()
        forms[form] = {"value": total_npm * nsteps / (ms / 1e3), "ms_per_step": ms / nsteps}
        tuned_by_form[form] = tuned

    # sequential plain runs, tuned by size class
    class_tuning = []
    seq_shape = {}
    if not args.no_autotune:
        counts = [p.par.npm for p in parts]
        for members in size_classes(counts):
            rep = members[int(np.argsort([counts[k] for k in members])[len(members) // 2])]
            p = parts[rep]
            s = lq.Simulation(p.par, *p.arrays())
            s.step(args.warmup)
            shape, skin = s.autotune(args.tune_steps)
            wide = s.wide_skin()
            s.close()
            for k in members:
                seq_shape[k] = (shape, skin, wide)
            class_tuning.append({"scenarios": len(members), "representative_npm": counts[rep],
                                 "pair_shape": shape, "skin_over_h": skin, "wide_over_h": wide})
    ms_seq = 0.0
    for k, p in enumerate(parts):
        s = lq.Simulation(p.par, *p.arrays())
        if k in seq_shape:
            s.set_pair_shape(seq_shape[k][0])
            s.set_skin(seq_shape[k][1])
            s.set_wide_skin(seq_shape[k][2])
        s.step(args.warmup)
        ms_seq += timed(s, nsteps)
        s.close()
    ms_seq = replicas.max_over_ranks(ms_seq, device="cuda")
    v_seq = total_npm * nsteps / (ms_seq / 1e3)
    out = {
        "workload": "ensemble of %d Drucker-Prager column collapses (counts log-uniform 5e3-2e5, H/L 0.5-4, "
                    "phi 20-40 deg, c 0-5 kPa, dr=2 mm, h=1.2dr)" % args.scenarios,
        "npm": total_npm, "rank0_np": par.np, "rank0_ncell": par.ncell, "steps": nsteps,
        "forms": forms,
        "sequential": {"value": v_seq, "ms_per_step": ms_seq / nsteps,
                       "form": "the same scenarios one after another, one plain FP32 simulation each, tuned by "
                               "size class", "tuning": class_tuning},
        "batched_over_sequential": {f: forms[f]["value"] / v_seq for f in forms},
        "autotuned": tuned_by_form,
        "partition": {"ranks": world, "imbalance": replicas.imbalance([p.par.npm for p in all_parts], shares)},
    }
    out.update(extra)
    return out


def bench_ensemble(args):
    """--config ensemble: the batched ensemble as the line's value."""
    import torch

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    m = ensemble_measurement(args, torch, world, rank, local, dist, sample_clocks=True)
    if rank == 0:
        v = m["forms"][args.form]
        print(json.dumps({
            "metric": "particle-steps/s", "value": v["value"], "unit": "particle-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": v["ms_per_step"],
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f32" if args.form == "plain" else "f32+f64", "data": "synthetic",
            "config": {"workload": m["workload"], "npm": m["npm"]},
            "form": "batched (%s): one simulation, per-scenario frames and materials, CUDA-graph step"
                    % ("mixed precision" if args.form == "mixed" else "plain FP32"),
            "forms": m["forms"], "sequential": m["sequential"],
            "batched_over_sequential": m["batched_over_sequential"][args.form],
            "autotuned": m["autotuned"], "gpu_launches_per_step": m["gpu_launches_per_step"],
            "neighbour_list_rebuilds": m["neighbour_list_rebuilds"],
            "neighbour_list_renewals": m["neighbour_list_renewals"], "health": m["health"],
            "phases_ms_per_step": m.get("phases_ms_per_step"),
            "clocks": m["clocks"], "partition": m["partition"],
        }))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main(argv=None):
    args = parse_args(argv)
    if args.impl == "reference":
        return bench_reference(args)
    if args.config == "ensemble":
        return bench_ensemble(args)
    return bench_ours(args)


if __name__ == "__main__":
    sys.exit(main())
