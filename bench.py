#!/usr/bin/env python
"""Benchmark of the ParaTC per-RK3-substep hot path on B200.

Metric: grid-point RK3 substeps/s = cells x substeps / device time, whole job.
Workload (default): the closed turbulent channel 128 x 96 x 128 (Re_b = 5600,
4pi x 2 x 4pi/3, tanh y-grid, RK3, dt = 0.005, constant flow rate, FP64),
seeded Poiseuille + U(-0.3, 0.3) noise made solenoidal by one projection.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One process per GPU (torchrun for N > 1); every rank advances its own channel
replica (weak scaling, no data-path collective); the timed region is
bracketed by a barrier and a device synchronisation and its length is the max
over ranks.  Between timed steps the L2 is flushed by writing a 256 MB buffer
(outside the events).  --impl reference times the CPU restatement of the
reference on all host cores (the reference itself, Fortran + MPI, cannot be
built on this image).
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "grid-point RK3 substeps/s"
UNIT = "grid-point substeps/s"
L2_BYTES = 126 * 1024 * 1024


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="channel_c1")
    ap.add_argument("--grid", type=int, nargs=3, default=None, metavar=("NX", "NY", "NZ"),
                    help="poisson_c2 and poisson_c2_zslabs: solve on this grid instead of 512 x 256 x 512")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the FP32 / mixed / batched forms that follow the FP64 headline")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--rhs-var", type=int, default=-1,
                    help="with --schedule: pin the right-hand-side launch shape too (paratc_tuning.rhs_var)")
    ap.add_argument("--helm-var", type=int, default=-1,
                    help="with --schedule: pin the Helmholtz launch shape too (paratc_tuning.helm_var)")
    ap.add_argument("--schedule", type=int, default=-1,
                    help="pin a Poisson schedule (0-11, paratc_set_schedule) instead of auto-tuning it")
    ap.add_argument("--batch-mode", choices=["grouped", "streams"], default="streams",
                    help="ensemble_c4: one launch per kernel instantiation over the members (grouped) or "
                         "every member's own launches on its own stream")
    ap.add_argument("--precision", choices=["fp64", "mixed", "fp32"], default="fp64",
                    help="mixed: the explicit right-hand side in FP32 arithmetic, all else FP64; "
                         "fp32: FP32 storage of everything but the pressure")
    return ap.parse_args()


def _case(name):
    from paratc_b200 import cases
    if name == "channel_c1":
        return cases.channel_c1()
    if name == "turbidity_c5":
        return cases.turbidity_c5()
    if name == "lock_exchange_c3":
        return cases.lock_exchange_c3()
    raise SystemExit("unknown workload " + name + " (ensemble_c4 has its own driver)")


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _traffic_table():
    """Per-launch DRAM bytes of ncu captures: profiles/ncu_traffic.txt lines
    '<workload> <kernel class> <bytes per launch>'."""
    out = {}
    p = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    if os.path.exists(p):
        for line in open(p):
            f = line.split()
            if len(f) == 3 and not line.startswith("#"):
                out[(f[0], f[1])] = float(f[2])
    return out


def algorithmic_bytes(params, precision="fp64"):
    """Compulsory HBM bytes per launch of each kernel class (N cells; spectral
    arrays hold (nx/2+1)*ny*nz complex values, S doubles).  FP64 and mixed
    forms: 8-byte words.  FP32 storage form: 4-byte velocity, scalar,
    histories, right-hand sides, potential and spectrum; the pressure stays
    8 bytes."""
    N = params.nxc * params.nyc * params.nzc
    S = 2 * (params.nxc // 2 + 1) * params.nyc * params.nzc  # doubles in the spectral array
    sc = 1 if params.scalar_on else 0
    w = 4 if precision == "fp32" else 8
    wp = 8  # the pressure
    return {
        "rhs": (12 + 4 * sc) * w * N + wp * N,    # u,v,w,p,H* in; Rhs*,H* out
        "helmholtz": 9 * w * N,                   # Rhs*, u* in; u* out
        "helmholtz_scalar": 3 * w * N,
        "prsrc": w * (3 * N + S),                 # u,v,w in; x spectrum out (source fused into the x transform)
        "fft_x_fwd": w * (N + S),
        "fft_z_fwd": 2 * w * S,
        "ysolve": 2 * w * S,
        "fft_z_bwd": 2 * w * S,
        "fft_x_bwd": w * (S + N),
        "project": 7 * w * N + 2 * wp * N,        # phi,u,v,w,p in; u,v,w,p out
        "cfl": 3 * w * N,
        "check": (3 + sc) * w * N,
    }


def kernel_fractions(prof, alg, peak):
    """Fraction of the HBM peak that every kernel class reaches: its
    compulsory bytes per launch (algorithmic_bytes) over its mean event time,
    divided by the measured peak (GB/s).  prof: {class: (total ms, launches)}."""
    out = {}
    for k, (ms_tot, n) in sorted(prof.items(), key=lambda kv: -kv[1][0]):
        if k in alg and n > 0 and ms_tot > 0:
            out[k] = round(alg[k] / (ms_tot / n / 1e3) / 1e9 / peak, 3)
    return out


class ClockSampler:
    """nvidia-smi clocks and throttle reasons every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                self.rows.append(f)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(self.rows)}


def _set_schedule(ctx, args):
    """The Poisson schedule: auto-tuned (5 solves per choice) unless pinned;
    returns the choice and the tuner's ms per 5 solves (-1: unsupported)."""
    if args.schedule >= 0:
        ctx.schedule = args.schedule
        return args.schedule, None
    choice, times = ctx.autotune(nrep=5)
    return choice, [round(float(t), 4) for t in times]


def _tune_step(ctx, args):
    """The channel workloads: the Poisson schedule and the right-hand-side and
    Helmholtz launch shapes, each combination timed as whole steps from a
    snapshot of the state (paratc_autotune_all), unless the schedule is
    pinned.  Returns the schedule and the picks."""
    if args.schedule >= 0:
        ctx.schedule = args.schedule
        if args.rhs_var >= 0 or args.helm_var >= 0:
            t = ctx.tuning
            if args.rhs_var >= 0:
                t.rhs_var = args.rhs_var
            if args.helm_var >= 0:
                t.helm_var = args.helm_var
            ctx.tuning = t
        return args.schedule, None
    t = ctx.autotune_all(nrep=3)
    return t.schedule, {"schedule": t.schedule, "rhs_var": t.rhs_var, "helm_var": t.helm_var,
                        "step_ms": round(t.step_ms, 4)}


def _dist():
    from paratc_b200.replicas import dist_env
    return dist_env()


def cpu_baseline(case, yp, fields, seconds, max_steps=200):
    """The oracle (CPU restatement of the reference) on all host threads."""
    from oracle import oracle_lib as ol
    threads = os.cpu_count() or 1
    o = ol.Oracle(case.params, yp, threads=threads)
    o.set_fields(fields["ux"], fields["uy"], fields["uz"], fields["p"], fields["c"])
    o.project()
    o.step()  # warm-up
    n = 0
    t0 = time.perf_counter()
    while True:
        o.step()
        n += 1
        el = time.perf_counter() - t0
        if el >= seconds or n >= max_steps:
            break
    o.close()
    iad = {1: 1, 2: 2, 3: 3}[case.params.ischeme]
    return {"value": case.n_cells * iad * n / el, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": "%d full RK3 steps of %s on the C oracle (OpenMP, %d threads), %.1f s" % (n, case.name, threads, el)}


def run_reference_poisson(args):
    """The reference arm of the Poisson workloads: the oracle's clcPPE (FFTW-
    style halfcomplex transforms and the Thomas sweeps, OpenMP over all host
    threads) on the same grid and source, `steps` solves after `warmup`."""
    from paratc_b200 import cases
    from oracle import oracle_lib as ol
    case = cases.poisson_c2(*args.grid) if args.grid else cases.poisson_c2()
    p = case.params
    m = case.mesh
    yp = ol.ycoord(m.section_length, m.section_cstret, m.nyc_section, m.stret_type, m.stret_option, p.yly)
    src = cases.gaussian_source(cases.Case("src", p, case.mesh, "gauss_src", 42, 1.0))
    threads = os.cpu_count() or 1
    o = ol.Oracle(p, yp, threads=threads)
    for _ in range(args.warmup):
        o.poisson(src)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o.poisson(src)
    el = time.perf_counter() - t0
    o.close()
    cells = p.nxc * p.nyc * p.nzc
    val = cells * args.steps / el
    unit = "grid-point Poisson solves/s"
    line = {"impl": "reference", "metric": unit, "value": val, "unit": unit, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
            "higher_is_better": True, "scaling": "strong" if args.workload.endswith("zslabs") else "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": case.name + ("_zslabs" if args.workload.endswith("zslabs") else ""),
                       "grid": [p.nxc, p.nyc, p.nzc], "precision": "fp64", "parallelism": "host threads"},
            "cpu_baseline": {"value": val, "unit": unit, "cores": threads, "kind": "port",
                             "sample": "%d Poisson solves of %s on the C oracle (OpenMP, %d threads)"
                                       % (args.steps, case.name, threads)},
            "e2e": {"value": val, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_reference(args):
    ws, rank, _ = _dist()
    if rank != 0:
        return
    if args.workload in ("poisson_c2", "poisson_c2_zslabs"):
        run_reference_poisson(args)
        return
    from paratc_b200 import cases
    from oracle import oracle_lib as ol
    case = _case(args.workload)
    m = case.mesh
    yp = ol.ycoord(m.section_length, m.section_cstret, m.nyc_section, m.stret_type, m.stret_option, case.params.yly)
    fields = cases.initial_fields(case, yp)
    threads = os.cpu_count() or 1
    o = ol.Oracle(case.params, yp, threads=threads)
    o.set_fields(fields["ux"], fields["uy"], fields["uz"], fields["p"], fields["c"])
    o.project()
    for _ in range(args.warmup):
        o.step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o.step()
    el = time.perf_counter() - t0
    iad = {1: 1, 2: 2, 3: 3}[case.params.ischeme]
    val = case.n_cells * iad * args.steps / el
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": case.name, "grid": [case.params.nxc, case.params.nyc, case.params.nzc],
                       "scheme": "RK3", "precision": "fp64", "parallelism": "host threads"},
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": "%d full RK3 steps of %s on the C oracle (OpenMP, %d threads)" % (args.steps, case.name, threads)},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    from paratc_b200 import replicas
    dist = replicas.init("nccl")
    from paratc_b200 import cases
    from paratc_b200.lib import ChannelSystem, mesh_ycoord
    case = _case(args.workload)
    case.seed = replicas.replica_seed(case.seed, rank)
    p = case.params
    yp = mesh_ycoord(case.mesh, p.yly)
    fields = cases.initial_fields(case, yp)
    base = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        base = cpu_baseline(case, yp, fields, args.cpu_seconds)

    ctx = ChannelSystem(p, yp, device=local)
    ctx.precision = args.precision
    ctx.set_fields(fields["ux"], fields["uy"], fields["uz"], fields["p"], fields["c"])
    ctx.project()
    # InitPoissonSolver's auto-tuning (src/m_Poisson.f90:50-175), widened to
    # the launch shapes, before timing
    schedule, tune_ms = _tune_step(ctx, args)
    stream = torch.cuda.ExternalStream(ctx.stream, device=local)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=local)
    iad = {1: 1, 2: 2, 3: 3}[p.ischeme]

    for _ in range(args.warmup):
        ctx.iterate_async(1)
    ctx.last_diag()
    torch.cuda.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def timed_pass(profile):
        if profile:
            ctx.profile(True)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        l0 = ctx.launches
        for i in range(args.steps):
            with torch.cuda.stream(stream):
                flush.add_(1.0)
            ev[i][0].record(stream)
            ctx.iterate_async(1)
            ev[i][1].record(stream)
        d = ctx.last_diag()
        torch.cuda.synchronize()
        launches = ctx.launches - l0
        ms = [a.elapsed_time(b) for a, b in ev]
        prof = ctx.profile_read() if profile else None
        if profile:
            ctx.profile(False)
        return ms, d, launches, prof

    barrier()
    sampler = ClockSampler(local)
    sampler.start()
    ms, diag, launches, _ = timed_pass(False)
    clocks = sampler.stop()
    barrier()
    total_ms = replicas.max_over_ranks(sum(ms), dist, device=local)
    value = ws * p.nxc * p.nyc * p.nzc * iad * args.steps / (total_ms / 1e3)

    # per-kernel timing pass (same workload, events around every launch)
    _, _, _, prof = timed_pass(True)
    barrier()

    # end to end through the C ABI with host buffers (pinned)
    e2e = None
    if not args.no_e2e:
        # the state a step consumes and produces: u, v, w, p (and the scalar);
        # the explicit histories only for AB2, whose first substep reads the
        # previous step's (RK2/RK3 start with zeta_1 = 0, and the reference
        # restarts them without history, src/m_IOAndVisu.f90:485)
        names = ["ux", "uy", "uz", "p"] + (["c"] if p.scalar_on else [])
        if p.ischeme == 1:
            names += ["hx", "hy", "hz"] + (["hc"] if p.scalar_on else [])
        host = {n: torch.empty(ctx.shape, dtype=torch.float64, pin_memory=True).numpy() for n in names}
        cur = ctx.get_fields(names)
        for n in names:
            host[n][...] = cur[n]
        nbytes = sum(host[n].nbytes for n in names)
        t_e2e = 0.0
        barrier()
        for i in range(args.steps):
            with torch.cuda.stream(stream):
                flush.add_(1.0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ctx.set_fields(host["ux"], host["uy"], host["uz"], host["p"], host.get("c"), host.get("hx"), host.get("hy"),
                           host.get("hz"), host.get("hc"))
            ctx.iterate(1)
            ctx.get_fields_into(host)
            t_e2e += time.perf_counter() - t0
        t_e2e = replicas.max_over_ranks(t_e2e, dist, device=local)
        e2e = {"value": ws * p.nxc * p.nyc * p.nzc * iad * args.steps / t_e2e, "unit": UNIT,
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes + 12 * 8,
               "note": "per step: paratc_set_fields (%s from pinned host) + paratc_step + paratc_get_fields (same to host)"
                       % ",".join(names)}

    # the mixed form against the FP64 path: the same initial fields advanced by
    # the same number of steps (warm-up, timed, profiled, end to end)
    mixed_err = None
    if args.precision in ("mixed", "fp32"):
        nsteps = args.warmup + 2 * args.steps + (0 if args.no_e2e else args.steps)
        ref = ChannelSystem(p, yp, device=local)
        ref.set_fields(fields["ux"], fields["uy"], fields["uz"], fields["p"], fields["c"])
        ref.project()
        ref.iterate(nsteps)
        fr, fm = ref.get_fields(), ctx.get_fields()
        mixed_err = {"steps": nsteps}
        for n in ("ux", "uy", "uz", "p", "c"):
            if fr.get(n) is not None:
                mixed_err[n] = float(np.abs(fm[n] - fr[n]).max() / np.abs(fr[n]).max())
        ref.close()

    # the north star's forms on the same workload and box: the FP32 storage
    # form and the mixed form against the FP64 path (device time of K steps
    # after W warm-up steps, L2 flushed between steps, max over ranks; field
    # error against an FP64 context advanced the same W + K steps from the
    # same projected state), and the batched C4 ensemble
    forms = None
    if not args.no_forms and args.precision == "fp64":
        forms = {"fp64": {"value": value, "ms_per_step": total_ms / args.steps}}
        ref = ChannelSystem(p, yp, device=local)
        ref.set_fields(fields["ux"], fields["uy"], fields["uz"], fields["p"], fields["c"])
        ref.project()
        ref.iterate(args.warmup + args.steps)
        fr = ref.get_fields()
        ref.close()
        for form in ("fp32", "mixed"):
            c2 = ChannelSystem(p, yp, device=local)
            c2.schedule = schedule
            c2.set_fields(fields["ux"], fields["uy"], fields["uz"], fields["p"], fields["c"])
            c2.project()
            c2.precision = form
            _, tune2 = _tune_step(c2, args)  # the form's own launch shapes
            st2 = torch.cuda.ExternalStream(c2.stream, device=local)
            for _ in range(args.warmup):
                c2.iterate_async(1)
            c2.last_diag()
            barrier()
            evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
            for a, b in evs:
                with torch.cuda.stream(st2):
                    flush.add_(1.0)
                a.record(st2)
                c2.iterate_async(1)
                b.record(st2)
            d2 = c2.last_diag()
            torch.cuda.synchronize()
            ms2 = replicas.max_over_ranks(sum(a.elapsed_time(b) for a, b in evs), dist, device=local)
            fm = c2.get_fields()
            err = {"steps": args.warmup + args.steps}
            for n in ("ux", "uy", "uz", "p", "c"):
                if fr.get(n) is not None:
                    err[n] = float(np.abs(fm[n] - fr[n]).max() / np.abs(fr[n]).max())
            v2 = ws * p.nxc * p.nyc * p.nzc * iad * args.steps / (ms2 / 1e3)
            forms[form] = {"value": v2, "ms_per_step": ms2 / args.steps, "speedup_vs_fp64": v2 / value, "tuning": tune2,
                           "divmax_last_step": d2.divmax, "field_rel_err_vs_fp64_path": err}
            c2.close()
        # the C4 ensemble: member launches on member streams (FP64 and the FP32
        # storage form), and the grouped launches (FP64)
        for key, prec, mode in (("batched_c4", "fp64", "streams"), ("batched_c4_fp32", "fp32", "streams"),
                                ("batched_c4_grouped", "fp64", "grouped")):
            ens = ensemble_measure(args, local, dist, prec, steps=max(3, args.steps // 2), mode=mode)
            ens.pop("_batch").close()
            ens.pop("_cases")
            ens.pop("clocks", None)
            ens["speedup_vs_fp64_single"] = ens["value"] / value
            forms[key] = ens
        forms["batched_c4_grouped"]["speedup_vs_streams"] = (forms["batched_c4_grouped"]["value"]
                                                             / forms["batched_c4"]["value"])

    # roofline of the dominant kernel
    peak, peak_kind = _peaks()
    alg = algorithmic_bytes(p, args.precision)
    dom = max(prof.items(), key=lambda kv: kv[1][0])
    kname, (kms, kn) = dom
    avg_s = kms / kn / 1e3
    ach = alg[kname] / avg_s / 1e9
    tkey = ("fp32_" + kname) if args.precision == "fp32" else kname
    traffic = _traffic_table().get((args.workload, tkey))
    share = {k: round(v[0] / sum(x[0] for x in prof.values()), 4) for k, v in sorted(prof.items(), key=lambda kv: -kv[1][0])}
    roof = {"bound": "hbm", "kernel": kname, "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
            "frac": round(ach / peak, 4), "traffic": traffic, "peak_kind": peak_kind,
            "algorithmic_bytes_per_launch": alg[kname], "avg_launch_us": round(avg_s * 1e6, 2),
            "kernel_share": share, "kernel_frac": kernel_fractions(prof, alg, peak)}
    # whole-substep algorithmic bandwidth (every kernel's compulsory bytes / step time)
    step_bytes = sum(alg[k] * v[1] for k, v in prof.items() if k in alg) / args.steps
    roof["step_algorithmic_GBps"] = round(step_bytes / (statistics.mean(ms) / 1e3) / 1e9, 1)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": {"fp64": "f64", "mixed": "f32 rhs + f64", "fp32": "f32 storage + f64 pressure"}[args.precision],
                "data": "synthetic",
                "config": {"workload": case.name, "grid": [p.nxc, p.nyc, p.nzc], "scheme": "RK3",
                           "precision": args.precision, "parallelism": "replicas x%d" % ws,
                           "l2": "flushed between timed steps (256 MB write outside the events)",
                           "divmax_last_step": diag.divmax, "poisson_schedule": schedule, "tuning": tune_ms,
                           "field_rel_err_vs_fp64_path": mixed_err},
                "roofline": roof, "cpu_baseline": base, "e2e": e2e, "gpu_launches": launches, "clocks": clocks,
                "forms": forms}
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def ensemble_measure(args, local, dist, precision, steps=None, mode="streams"):
    """The C4 ensemble: 32 channel instances of uneven grids and Re_tau
    advanced together by the batch API, every step-round one CUDA graph
    launch (device time of `steps` steps, max over ranks); and the same
    instances stepped one after another, each alone on the GPU.  mode
    "grouped": one launch per kernel instantiation and stage over all members
    (paratc_batch_set_mode); "streams": every member's own launches on its
    own stream.  The ensemble's working set (several GB) exceeds the L2, so
    no flush is needed between timed steps.  Returns the measurement as a
    dict (with the batch and its cases under "_batch" and "_cases" for the
    caller to close)."""
    import torch
    from paratc_b200 import cases, replicas
    from paratc_b200.lib import BatchSystem, mesh_ycoord
    ws, rank, _ = _dist()
    steps = steps or args.steps
    cs = cases.ensemble_c4(seed=replicas.replica_seed(2024, rank))
    yps = [mesh_ycoord(c.mesh, c.params.yly) for c in cs]
    b = BatchSystem([c.params for c in cs], yps, device=local)
    cells = 0
    for c, y, m in zip(cs, yps, b.members):
        f = cases.initial_fields(c, y)
        m.set_fields(f["ux"], f["uy"], f["uz"], f["p"], f["c"])
        m.project()
        m.precision = precision
        cells += c.params.nxc * c.params.nyc * c.params.nzc
    b.mode = mode
    stream = torch.cuda.ExternalStream(b.stream, device=local)
    b.iterate(args.warmup)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    diags = b.iterate(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = replicas.max_over_ranks(e0.elapsed_time(e1), dist, device=local)
    value = ws * cells * 3 * steps / (ms / 1e3)
    # the same members one at a time, each alone on the GPU
    seq_ms = 0.0
    for m in b.members:
        st = torch.cuda.ExternalStream(m.stream, device=local)
        a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        m.iterate_async(steps)
        z.record(st)
        m.last_diag()
        torch.cuda.synchronize()
        seq_ms += a.elapsed_time(z)
    seq_ms = replicas.max_over_ranks(seq_ms, dist, device=local)
    seq_value = ws * cells * 3 * steps / (seq_ms / 1e3)
    return {"value": value, "unit": UNIT, "ms_per_step": ms / steps, "steps": steps, "cells": cells,
            "precision": precision, "mode": mode, "graph_kernels_per_step": b.graph_kernels,
            "divmax_last_step_max": max(d.divmax for d in diags),
            "sequential": {"value": seq_value, "ms_per_step": seq_ms / steps,
                           "note": "the same 32 instances stepped one after another, each alone on the GPU"},
            "speedup_vs_sequential": value / seq_value, "clocks": clocks, "_batch": b, "_cases": cs}


def run_ensemble(args):
    """The C4 ensemble line (ensemble_measure), with the end-to-end figure:
    every member's state in from pinned host memory, one batch step, every
    member's state back."""
    import torch
    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    from paratc_b200 import replicas
    dist = replicas.init("nccl")
    r = ensemble_measure(args, local, dist, args.precision, mode=args.batch_mode)
    b = r.pop("_batch")
    cs = r.pop("_cases")
    cells = r["cells"]
    names = ["ux", "uy", "uz", "p"]
    host = []
    nbytes = 0
    for c, m in zip(cs, b.members):
        h = {n: torch.empty(m.shape, dtype=torch.float64, pin_memory=True).numpy() for n in names}
        cur = m.get_fields(names)
        for n in names:
            h[n][...] = cur[n]
            nbytes += h[n].nbytes
        host.append(h)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    # every member on its own stream: its state in, one step, its state out;
    # the members' transfers and steps overlap one another
    t_e2e = 0.0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        for m, h in zip(b.members, host):
            m.set_fields_async(h["ux"], h["uy"], h["uz"], h["p"])
            m.iterate_async(1)
            m.get_fields_into_async(h)
        for m in b.members:
            m.sync()
        t_e2e += time.perf_counter() - t0
    for m in b.members:
        m.last_diag()
    t_e2e = replicas.max_over_ranks(t_e2e, dist, device=local)
    if rank == 0:
        line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": ws, "steps": r["steps"],
                "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": {"fp64": "f64", "mixed": "f32 rhs + f64", "fp32": "f32 storage + f64 pressure"}[args.precision],
                "data": "synthetic",
                "config": {"workload": "ensemble_c4: 32 channels, (nx,nz) in {64,96,128,192}, ny in {48,64,96,128}, "
                                       "Re_tau U[120,395], seed 2024",
                           "cells": cells, "precision": args.precision, "batch_mode": args.batch_mode,
                           "parallelism": "ensemble in one CUDA graph x%d" % ws,
                           "l2": "working set %.1f GB > L2, no flush" % (cells * 17 * 8 / 1e9),
                           "graph_kernels_per_step": r["graph_kernels_per_step"],
                           "divmax_last_step_max": r["divmax_last_step_max"]},
                "sequential": r["sequential"], "speedup_vs_sequential": r["speedup_vs_sequential"],
                "roofline": None, "cpu_baseline": None,
                "e2e": {"value": ws * cells * 3 * args.steps / t_e2e, "unit": UNIT, "h2d_bytes_per_step": nbytes,
                        "d2h_bytes_per_step": nbytes,
                        "note": "per step: every member's u,v,w,p from pinned host, one step, back; members pipelined "
                                "on their own streams (paratc_set_fields_async / steps_async / get_fields_async)"},
                "gpu_launches": r["graph_kernels_per_step"] * r["steps"], "clocks": r["clocks"]}
        print(json.dumps(line), flush=True)
    b.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_poisson(args):
    """C2: the standalone pressure Poisson solve, 512 x 256 x 512, seeded
    Gaussian right-hand side with its mean removed.  `value` in grid points
    solved per second; the roofline counts 6 words per cell (forward 2-D FFT,
    y-Thomas, inverse 2-D FFT, each a read and a write).  src and phi (537 MB
    each) exceed the L2, so no flush is needed between solves."""
    import torch
    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    from paratc_b200 import cases
    from paratc_b200.lib import ChannelSystem, mesh_ycoord
    case = cases.poisson_c2(*args.grid) if args.grid else cases.poisson_c2()
    p = case.params
    yp = mesh_ycoord(case.mesh, p.yly)
    src = cases.gaussian_source(cases.Case("src", p, case.mesh, "gauss_src", 42 + rank, 1.0))
    cells = p.nxc * p.nyc * p.nzc
    ctx = ChannelSystem(p, yp, device=local)
    schedule, tune_ms = _set_schedule(ctx, args)  # InitPoissonSolver's auto-tuning, before timing
    stream = torch.cuda.ExternalStream(ctx.stream, device=local)
    d_src = torch.from_numpy(src).to("cuda:%d" % local)
    d_phi = torch.empty_like(d_src)
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        ctx.poisson_device(d_src.data_ptr(), d_phi.data_ptr())
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    sampler = ClockSampler(local)
    sampler.start()
    for a, b in evs:
        a.record(stream)
        ctx.poisson_device_async(d_src.data_ptr(), d_phi.data_ptr())
        b.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = sum(a.elapsed_time(b) for a, b in evs)
    phi_g = d_phi.cpu().numpy()
    # per-kernel event times of the same solves
    ctx.profile(True)
    for _ in range(args.steps):
        ctx.poisson_device_async(d_src.data_ptr(), d_phi.data_ptr())
    torch.cuda.synchronize()
    prof = ctx.profile_read()
    ctx.profile(False)
    kern = {k: round(v[0] / max(v[1], 1) * 1e3, 1) for k, v in prof.items() if v[1] > 0}
    # end to end: host source in, host potential out (paratc_poisson)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        phi_h = ctx.poisson(src)
    t_e2e = time.perf_counter() - t0
    # the second form of this configuration: FP32 solves (spectrum stored in
    # FP32, FP64 arithmetic in the passes) with FP64-residual iterative
    # refinement to max|r| <= 1e-12 max|src|; the corrections needed are
    # counted once, then that many are timed per solve
    refined = None
    if not args.no_forms:
        d_phr = torch.empty_like(d_src)
        ncorr, relres = ctx.poisson_refined(d_src.data_ptr(), d_phr.data_ptr(), 1e-12, 4)
        evr = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for _ in range(args.warmup):
            ctx.poisson_refined_async(d_src.data_ptr(), d_phr.data_ptr(), ncorr)
        torch.cuda.synchronize()
        for a, b in evr:
            a.record(stream)
            ctx.poisson_refined_async(d_src.data_ptr(), d_phr.data_ptr(), ncorr)
            b.record(stream)
        torch.cuda.synchronize()
        msr = sum(a.elapsed_time(b) for a, b in evr)
        phr = d_phr.cpu().numpy()
        # bytes one refined solve moves (8-byte words per cell, spectrum S ~ N
        # doubles stored as floats): first solve 7 (FP64 source in, FP32
        # spectrum through x, z, y with FP64 pivots, z, x, FP64 potential
        # out), each correction 3 (residual: source, potential, r) + 8
        # (the same solve, potential read and written)
        words = 7 + 11 * ncorr
        refined = {"value": cells * args.steps / (msr / 1e3), "unit": "grid-point Poisson solves/s",
                   "ms_per_solve": msr / args.steps, "corrections": ncorr, "relres": relres,
                   "speedup_vs_fp64": ms / msr, "bytes_per_cell": 8 * words,
                   "GBps": 8 * words * cells / (msr / args.steps / 1e3) / 1e9}
    base = None
    err = None
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import oracle_lib as ol
        threads = os.cpu_count() or 1
        o = ol.Oracle(p, yp, threads=threads)
        t0 = time.perf_counter()
        phi_o = o.poisson(src)
        t_o = time.perf_counter() - t0
        o.close()
        err = float(np.abs(phi_g - phi_o).max() / np.abs(phi_o).max())
        if refined is not None:
            refined["rel_err_vs_oracle"] = float(np.abs(phr - phi_o).max() / np.abs(phi_o).max())
            refined["rel_err_vs_fp64_path"] = float(np.abs(phr - phi_g).max() / np.abs(phi_g).max())
        base = {"value": cells / t_o, "unit": "grid-point Poisson solves/s", "cores": threads, "kind": "port",
                "sample": "one %dx%dx%d solve on the C oracle (OpenMP, %d threads), %.1f s"
                          % (p.nxc, p.nyc, p.nzc, threads, t_o)}
    peak, peak_kind = _peaks()
    alg = 6 * 8 * cells
    ach = alg / (ms / args.steps / 1e3) / 1e9
    if rank == 0:
        line = {"metric": "grid-point Poisson solves/s", "value": ws * cells * args.steps / (ms / 1e3),
                "unit": "grid-point Poisson solves/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic",
                "config": {"workload": case.name, "grid": [p.nxc, p.nyc, p.nzc], "precision": "fp64",
                           "l2": "src and phi %d MB each%s, no flush" % (src.nbytes // 10**6, " > L2" if src.nbytes > L2_BYTES else ""),
                           "max_rel_err_vs_oracle": err, "poisson_schedule": schedule, "autotune_ms": tune_ms, "mean_phi_e2e_equal": bool(np.array_equal(phi_h, phi_g))},
                "roofline": {"bound": "hbm", "kernel": "poisson solve (5 kernels)", "achieved": round(ach, 1),
                             "peak": peak, "unit": "GB/s", "frac": round(ach / peak, 4), "traffic": None,
                             "peak_kind": peak_kind, "algorithmic_bytes_per_launch": alg,
                             "kernel_us": kern, "kernel_frac": kernel_fractions(prof, algorithmic_bytes(p), peak)},
                "cpu_baseline": base, "fp32_refined": refined,
                "e2e": {"value": cells * args.steps / t_e2e, "unit": "grid-point Poisson solves/s",
                        "h2d_bytes_per_step": src.nbytes, "d2h_bytes_per_step": src.nbytes,
                        "note": "paratc_poisson with host arrays: source in, potential out"},
                "gpu_launches": None, "clocks": clocks}
        print(json.dumps(line), flush=True)
    ctx.close()


def run_poisson_slabs(args):
    """C2's Poisson solve split over the ranks as z slabs (paratc_slab_*):
    every rank transforms its planes along x, an exchange gives it all
    planes of its x modes, it solves the z transforms and y-Thomas systems
    there, a second exchange returns the planes, and it transforms them back.
    Two forms of the exchange are timed: the peer form (the headline: the
    library's scatter / gather kernels store into and load from every rank's
    x-slab, mapped by CUDA IPC) and the all-to-all form (NCCL
    all_to_all_single; device copies with one rank).  Total work is fixed as
    N grows (strong scaling); `value` is grid points solved per second of
    the slowest rank.  Every rank also solves the whole grid on its own GPU
    (paratc_poisson_device) and reports the largest difference over its
    planes."""
    import torch
    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    dev = "cuda:%d" % local
    from paratc_b200 import cases, replicas, slabs
    from paratc_b200.lib import ChannelSystem, mesh_ycoord
    dist = replicas.init("nccl") if ws > 1 else None
    case = cases.poisson_c2(*args.grid) if args.grid else cases.poisson_c2()
    p = case.params
    yp = mesh_ycoord(case.mesh, p.yly)
    src = cases.gaussian_source(cases.Case("src", p, case.mesh, "gauss_src", 42, 1.0))  # one problem for all ranks
    cells = p.nxc * p.nyc * p.nzc
    plan = slabs.SlabPoisson(p, yp, rank, ws, device=local)
    d_src = torch.from_numpy(np.ascontiguousarray(src[plan.k0:plan.k0 + plan.nzl])).to(dev).reshape(-1)
    d_phi = torch.empty_like(d_src)
    buf, xslab = plan.buffers(torch, dev)
    if dist is not None:
        exchange = slabs.nccl_exchange()
    else:
        def exchange(s, r, sc, rc):
            slabs.LocalExchange.all_to_all([s], [r], [sc], [rc])
    st = torch.cuda.current_stream()

    def solve():
        plan.solve(d_src, d_phi, exchange, buf, xslab, stream=st.cuda_stream)

    for _ in range(args.warmup):
        solve()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(local)
    sampler.start()
    a.record(st)
    for _ in range(args.steps):
        solve()
    b.record(st)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    plan.sync(st.cuda_stream)
    ms = replicas.max_over_ranks(a.elapsed_time(b), dist, device=local)
    # stage times of one more solve (events between the stages)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
    ev[0].record(st); plan.forward(d_src, buf, st.cuda_stream)
    ev[1].record(st); exchange(buf, xslab, plan.send_counts, plan.recv_counts)
    ev[2].record(st); plan.middle(xslab, st.cuda_stream)
    ev[3].record(st); exchange(xslab, buf, plan.recv_counts, plan.send_counts)
    ev[4].record(st); plan.backward(buf, d_phi, st.cuda_stream)
    ev[5].record(st)
    torch.cuda.synchronize()
    stages = dict(zip(["forward_x", "exchange_1", "middle_zyz", "exchange_2", "backward_x"],
                      [round(ev[i].elapsed_time(ev[i + 1]), 3) for i in range(5)]))
    phi_local = d_phi.cpu().numpy().reshape(plan.nzl, p.nyc, p.nxc)
    # the one-GPU solve of the whole grid on this rank's GPU
    ctx = ChannelSystem(p, yp, device=local)
    g_src = torch.from_numpy(src).to(dev)
    g_phi = torch.empty_like(g_src)
    torch.cuda.synchronize()
    ctx.poisson_device(g_src.data_ptr(), g_phi.data_ptr())
    ref = g_phi.cpu().numpy()
    ctx.close()
    err = float(np.abs(phi_local - ref[plan.k0:plan.k0 + plan.nzl]).max() / np.abs(ref).max())
    err = replicas.max_over_ranks(err, dist, device=local)
    # the peer form: the scatter kernel stores every value into its owner's
    # x-slab (IPC-mapped across processes), the gather kernel loads it back;
    # no collective library on the data path
    peer, why = None, None
    if dist is None:
        def peer_solve(out):
            slabs.LocalPeers.solve([plan], [d_src], [out], stream=st.cuda_stream)
    else:
        try:
            peer = slabs.PeerExchange(plan, dist, stream=st.cuda_stream)
        except Exception as e:  # every rank learns whether all ranks mapped their peers
            why = "peer mapping failed on rank %d: %s" % (rank, e)
        ok = replicas.max_over_ranks(0.0 if peer is not None else 1.0, dist, device=local) == 0.0

        def peer_solve(out):
            peer.solve(d_src, out)
        if not ok:
            peer_solve = None
    peer_line = None
    if peer_solve is not None:
        d_phi2 = torch.empty_like(d_src)
        for _ in range(args.warmup):
            peer_solve(d_phi2)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        a.record(st)
        for _ in range(args.steps):
            peer_solve(d_phi2)
        b.record(st)
        torch.cuda.synchronize()
        plan.sync(st.cuda_stream)
        ms_p = replicas.max_over_ranks(a.elapsed_time(b), dist, device=local)
        same = float(np.array_equal(d_phi2.cpu().numpy().reshape(plan.nzl, p.nyc, p.nxc), phi_local))
        same = replicas.max_over_ranks(1.0 - same, dist, device=local) == 0.0
        peer_line = {"value": cells * args.steps / (ms_p / 1e3), "ms_per_step": ms_p / args.steps,
                     "bitwise_equal_to_all_to_all_form": bool(same),
                     "exchange": "scatter / gather kernels into IPC-mapped x-slabs" if dist is not None
                                 else "scatter / gather kernels (one rank)"}
        if peer is not None:
            peer.close()
    nccl_line = {"value": cells * args.steps / (ms / 1e3), "ms_per_step": ms / args.steps,
                 "exchange": "NCCL all_to_all_single" if dist is not None else "device copies (one rank)",
                 "stages_ms_rank0": stages}
    head = peer_line if peer_line is not None else nccl_line
    if rank == 0:
        line = {"metric": "grid-point Poisson solves/s", "value": head["value"],
                "unit": "grid-point Poisson solves/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": case.name + "_zslabs", "grid": [p.nxc, p.nyc, p.nzc], "ranks": ws,
                           "planes_rank0": plan.nzl, "modes_rank0": plan.nxl, "exchange": head["exchange"],
                           "l2": "src and phi exceed the L2 at one rank, no flush",
                           "max_rel_err_vs_one_gpu_solve": err},
                "peer_form": peer_line if peer_line is not None else {"unavailable": why},
                "all_to_all_form": nccl_line,
                "e2e": None, "gpu_launches": (5 if peer_line is not None else 7) * args.steps, "clocks": clocks}
        print(json.dumps(line), flush=True)
    plan.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_diagnostics(args):
    """The output-side kernels on C1 (128 x 96 x 128, fields after 20 steps):
    one clcStat accumulation, one 1-D spectra sample (x and z), one 2-D
    spectra sample at 9 rows (+ mirrored rows), and every dump_visu quantity
    at all points, each timed with CUDA events on the context's stream over
    `steps` calls after `warmup` calls.  Reports microseconds per call and the
    HBM rate of the algorithmic bytes (each field read once, the output
    written once)."""
    import torch
    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    from paratc_b200 import cases
    from paratc_b200.abi import VISU_NAMES
    from paratc_b200.lib import ChannelSystem, mesh_ycoord
    case = cases.channel_c1()
    p = case.params
    yp = mesh_ycoord(case.mesh, p.yly)
    f = cases.initial_fields(case, yp)
    ctx = ChannelSystem(p, yp, device=local)
    ctx.set_fields(f["ux"], f["uy"], f["uz"], f["p"])
    ctx.project()
    ctx.iterate(20)
    stream = torch.cuda.ExternalStream(ctx.stream, device=local)
    cells = p.nxc * p.nyc * p.nzc
    out = torch.empty(cells, dtype=torch.float64, device="cuda:%d" % local)
    iy = [5, 10, 15, 20, 25, 30, 35, 40, 45]
    ctx.spectra2d_setup(iy)
    calls = {
        "stats": (lambda: ctx.stats_accumulate(), 4 * 8 * cells),
        "spectra_1d": (lambda: ctx.spectra_accumulate(20), 2 * 6 * 8 * cells),
        "spectra_2d_9rows": (lambda: ctx.spectra2d_accumulate(), 6 * 2 * len(iy) * 8 * p.nxc * p.nzc * 3),
    }
    for n in VISU_NAMES:
        if n == "scalar":
            continue
        nread = 1 if n in ("ux", "uy", "uz", "pr") else 3
        calls["visu_" + n] = ((lambda n=n: ctx.visu_quantity_device_async(n, out.data_ptr())), (nread + 1) * 8 * cells)
    res = {}
    for name, (fn, alg) in calls.items():
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.steps):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        us = a.elapsed_time(b) / args.steps * 1e3
        res[name] = {"us_per_call": round(us, 1), "alg_GBs": round(alg / (us * 1e-6) / 1e9, 1)}
    ctx.spectra_reset()
    ctx.stats_reset()
    if rank == 0:
        peak, peak_kind = _peaks()
        print(json.dumps({"metric": "diagnostic call time", "workload": case.name, "unit": "us per call",
                          "grid": [p.nxc, p.nyc, p.nzc], "steps": args.steps, "warmup": args.warmup,
                          "peak_GBs": peak, "peak_kind": peak_kind, "calls": res}), flush=True)
    ctx.close()


def main():
    args = _args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "ensemble_c4":
        run_ensemble(args)
    elif args.workload == "poisson_c2":
        run_poisson(args)
    elif args.workload == "poisson_c2_zslabs":
        run_poisson_slabs(args)
    elif args.workload == "diagnostics_c1":
        run_diagnostics(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
