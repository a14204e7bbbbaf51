#!/usr/bin/env python
"""Throughput of the f(R) particle-mesh step on B200: particle-steps per second.

Workload (default): f(R) Hu-Sawicki F5 (|f_R0| = 1e-5, n = 1), flat LCDM
(Om = 0.3089, OmL = 0.6911, h = 0.6774, n_s = 0.9667, sigma8 = 0.8159),
Np = 512^3 particles on a 1024^3 mesh, L = 1024 Mpc/h, Zel'dovich initial
conditions at a = 0.02 from a seeded Gaussian random field (seed 7), 100-step
schedule.  A step is one pass of the reference's main loop (PMP2main.f90:36-60):
CIC density, MG scalar-field solve (V-cycles, residual target 1e-8, at most 4
cycles), FFT Poisson solve, fifth-force coupling, kick and drift.  The timed
steps are steps 1..K of the schedule from a = 0.02 (K = 100 runs it to z = 0),
after W untimed warm-up steps.

The timed form is the precision form (MGG_PREC_MIXED) unless --precision plain:
the metric is throughput at a P(k) error below 1e-3 against the plain GPU path,
so the plain drop-in path is timed over the same steps from the same initial
conditions and the line reports both and the P(k) error between them.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--precision mixed|plain]

With N > 1 (torchrun) every rank advances its own box (replicas: the PM step
of one box does not shard); the value is all ranks' particle-steps over the
slowest rank's device time.  `--impl reference` times the CPU restatement of
the reference (oracle/, C++ + OpenMP on all host cores) on the same workload:
step 1 of the schedule at full size from numpy Zel'dovich initial conditions
(--ref-steps of them; each takes minutes of host work at 512^3 / 1024^3).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "mg-glam-durham_b200"))

METRIC = "f(R) PM particle-steps/s"


def metric_of(workload: str) -> str:
    """The headline metric for f(R); the same metric named for the other solvers."""
    model = WORKLOADS[workload]["model"]
    return METRIC if model == "fr" else {"dgp": "nDGP", "sym": "symmetron", "kmf": "k-mouflage"}[model] + " PM particle-steps/s"
UNIT = "particle-steps/s"

# The single-box workloads: f(R) F5 (the headline 512^3 / 1024^3 run, a smaller
# one and the CPU-runnable 128^3 / 256^3 setup) and the other solvers at
# 512^3 particles on a 1024^3 mesh, L = 512 Mpc/h, seed 11, 100 steps.
WORKLOADS = {
    "fr5_512_1024": dict(nrow=512, ngrid=1024, box=1024.0, seed=7, nsteps=100, model="fr"),
    "fr5_256_512": dict(nrow=256, ngrid=512, box=512.0, seed=7, nsteps=100, model="fr"),
    "fr5_128_256": dict(nrow=128, ngrid=256, box=256.0, seed=42, nsteps=40, model="fr"),
    "dgp_512_1024": dict(nrow=512, ngrid=1024, box=512.0, seed=11, nsteps=100, model="dgp"),
    "sym_512_1024": dict(nrow=512, ngrid=1024, box=512.0, seed=11, nsteps=100, model="sym"),
    "kmf_512_1024": dict(nrow=512, ngrid=1024, box=512.0, seed=11, nsteps=100, model="kmf"),
}
MODELS = {   # model code, description (the parameters are the config defaults of make_config)
    "fr": (1, "f(R) Hu-Sawicki F5 (fR0=-1e-5, n=1)"),
    "dgp": (2, "nDGP normal branch, H0 rc = 1"),
    "sym": (3, "symmetron a*=0.5, beta=1, lambda_phi=1 Mpc/h"),
    "kmf": (4, "k-mouflage K(X) = -1 + X + K0 X^3, K0=1, beta=0.1"),
}
PRECISION_DOC = {
    "mixed": "precision form MGG_PREC_MIXED: smoother updates in FP32 (f(R) / symmetron roots by FP32 Newton from "
             "the cell's value, FP64 closed form where that start is unusable); FP32 residuals, FAS right-hand sides "
             "and prolongation (f(R) n=1 also the level-1 restriction) with FP64 norm accumulation; CIC, FFT, "
             "coupling and MOVE as the plain path; P(k) checked against the plain path",
    "plain": "plain drop-in path MGG_PREC_PLAIN: FP32 storage, FP64 arithmetic where the reference uses Real*8",
}
COSMO = dict(om=0.3089, oml=0.6911, omb=0.0486, hubble=0.6774, ns=0.9667, sigma8=0.8159)
# mgg_mg_report.exit_reason: the exit tests of scalar_field (PMP2extradof.f90:107-121)
EXIT_REASONS = {0: "skipped (a < a*)", 1: "residual <= res_conv", 2: "stagnation", 3: "iter_count_max"}
A0 = 0.02


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kernel: str, workload: str):
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    return d.get(workload, {}).get(kernel)


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        if self.path and os.path.exists(self.path):
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


# ----------------------------------------------------------- CPU baseline ---
def numpy_ics(nrow, ngrid, boxsize, seed, aexpn, astep):
    """Zel'dovich initial conditions with numpy (input generation for the CPU arm only)."""
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((nrow, nrow, nrow))
    W = np.fft.rfftn(w)
    kf = np.fft.fftfreq(nrow, 1.0 / nrow)
    kr = np.fft.rfftfreq(nrow, 1.0 / nrow)
    mz, my, mx = np.meshgrid(kf, kf, kr, indexing="ij")
    m2 = mx ** 2 + my ** 2 + mz ** 2
    om, omb, h, ns, s8 = COSMO["om"], COSMO["omb"], COSMO["hubble"], COSMO["ns"], COSMO["sigma8"]
    gamma = om * h * np.exp(-omb * (1.0 + np.sqrt(2 * h) / om))

    def T(k):
        q = k / gamma
        with np.errstate(divide="ignore", invalid="ignore"):
            t = np.log(1 + 2.34 * q) / (2.34 * q) * (1 + 3.89 * q + (16.1 * q) ** 2 + (5.46 * q) ** 3 + (6.71 * q) ** 4) ** -0.25
        return np.where(q > 0, t, 1.0)

    lk = np.linspace(np.log(1e-5), np.log(1e3), 4001)
    k = np.exp(lk)
    x = k * 8.0
    Wt = 3 * (np.sin(x) - x * np.cos(x)) / x ** 3
    s2 = np.trapezoid(k ** 3 * k ** ns * T(k) ** 2 * Wt ** 2, lk) / (2 * np.pi ** 2)
    amp = s8 ** 2 / s2

    def E(a):
        return np.sqrt(om / a ** 3 + COSMO["oml"])

    def growth(a):
        xs = a * (np.arange(2000) + 0.5) / 2000
        return 2.5 * om * E(a) * np.sum(1.0 / (xs * E(xs)) ** 3) * a / 2000

    D = growth(aexpn) / growth(1.0)
    kphys = 2 * np.pi * np.sqrt(m2) / boxsize
    with np.errstate(divide="ignore", invalid="ignore"):
        P = np.where(m2 > 0, amp * kphys ** ns * T(kphys) ** 2, 0.0)
    P = np.where(np.sqrt(m2) >= nrow // 2, 0.0, P)
    delta = W * np.sqrt(P / (boxsize ** 3 * nrow ** 3)) * D
    qfact = ngrid / nrow
    parts = []
    vels = []
    aexpv = np.float32(aexpn - astep / 2)
    vfac = float(aexpv / np.float32(aexpn)) * np.sqrt(float(aexpv)) * np.sqrt(om + COSMO["oml"] * float(aexpv) ** 3)
    idx = np.arange(nrow)
    for comp, mc in enumerate((mx, my, mz)):
        with np.errstate(divide="ignore", invalid="ignore"):
            f = np.where(m2 > 0, 1j * mc / m2, 0.0) * ngrid / (2 * np.pi)
        d = np.fft.irfftn(delta * f, s=(nrow, nrow, nrow), axes=(0, 1, 2)) * nrow ** 3
        lat = np.meshgrid(idx, idx, idx, indexing="ij")[2 - comp]
        xq = (qfact * lat + 1.0 + 0.5 + d).astype(np.float32)
        xq = np.where(xq > ngrid + 1, xq - ngrid, xq)
        xq = np.where(xq <= 1.0, xq + ngrid, xq)
        xq = np.where(xq >= ngrid + 1, xq - np.float32(1e-3), xq).astype(np.float32)
        parts.append(np.ascontiguousarray(xq).reshape(-1))
        vels.append(np.ascontiguousarray((d * vfac).astype(np.float32)).reshape(-1))
    return parts + vels


def cpu_step(orc, cfg, st, fi2, parts, i, nthreads, bg=None):
    """One main-loop step (PMP2main.f90:36-60) on the CPU restatement."""
    f32 = np.float32
    N = cfg.ngrid
    fi = orc.density(parts[0], parts[1], parts[2], N, nthreads=nthreads)
    fi2, rep = orc.scalar_field(fi, fi2, cfg, st["a"], i, nthreads=nthreads, bg=bg)
    phi = orc.potential(fi, N, st["a"], cfg.om, cfg.omb, nthreads=nthreads)
    factv = f32(1.0)
    if f32(st["da"]) < f32(f32(st["sf"]) / f32(1.25)) * f32(st["a"]) and f32(st["a"]) < f32(0.3):
        st["da"] = float(f32(f32(1.5) * f32(st["da"])))
        factv = f32(1.2)
    phi = orc.potential_mg(phi, fi2, cfg, st["a"], nthreads=nthreads)
    parts, ekin = orc.move(phi, fi2, parts, cfg, st["a"], st["da"], float(factv), bg=bg, nthreads=nthreads)
    st["a"] = float(f32(f32(st["a"]) + f32(st["da"])))
    return fi2, parts


def run_cpu(steps: int, warmup: int, workload: str = "fr5_512_1024"):
    """The oracle port on all host threads: (particle-steps/s, cores, sample).  The
    sample is 128^3 particles on a 256^3 mesh of the workload's model and cell size,
    on the workload's 100-step schedule."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import mgglam_b200 as m
    import oracle as orc

    full = WORKLOADS[workload]
    w = dict(WORKLOADS["fr5_128_256"], box=256.0 * full["box"] / full["ngrid"])
    model, mdesc = MODELS[full["model"]]
    nt = os.cpu_count() or 1
    astep0 = m.astep_for_nsteps(A0, full["nsteps"])
    cfg = m.make_config(w["ngrid"], w["nrow"], w["box"], om=COSMO["om"], oml=COSMO["oml"], omb=COSMO["omb"],
                        mg_model=model, fr_n=1, fr0=-1e-5)
    bg = m.background_table(cfg)[0] if model in (m.MODEL_KMOUFLAGE, m.MODEL_CSF) else None
    parts0 = numpy_ics(w["nrow"], w["ngrid"], w["box"], w["seed"], A0, astep0)

    def fresh():
        return ([a.copy() for a in parts0], {"a": A0, "da": astep0, "sf": float(np.float32(np.float32(astep0) / np.float32(A0)))},
                np.zeros(w["ngrid"] ** 3, np.float32))

    parts, st, fi2 = fresh()
    for i in range(1, warmup + 1):
        fi2, parts = cpu_step(orc, cfg, st, fi2, parts, i, nt, bg)
    # timed: steps 1..K of the schedule from the initial conditions, as the GPU arm
    parts, st, fi2 = fresh()
    t0 = time.perf_counter()
    for i in range(1, steps + 1):
        fi2, parts = cpu_step(orc, cfg, st, fi2, parts, i, nt, bg)
    dt = time.perf_counter() - t0
    npart = w["nrow"] ** 3
    sample = (f"steps 1..{steps} of the 128^3-particle / 256^3-mesh (L = {w['box']:g} Mpc/h) {mdesc} "
              f"{full['nsteps']}-step schedule from a={A0} (the particles per cell, cell size and per-particle work "
              f"of {full['nrow']}^3/{full['ngrid']}^3), C++/OpenMP restatement, {nt} threads")
    return npart * steps / dt, nt, sample, dt / steps * 1e3


# ------------------------------------------------------------- GPU arm ----
def dist_setup(n_gpus):
    """One process per GPU (torchrun): NCCL with a CUDA device, gloo without (CPU tests).
    Replicas only: each rank advances its own box; the only collectives are the
    barrier and the max over ranks of the timed region."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def replica_seed(base: int, rank: int) -> int:
    """Each rank's box is an independent realisation (PMP2mainMPI.f90:27-30)."""
    return base + rank


def aggregate_value(npart: int, steps: int, world: int, ms_max: float) -> float:
    """Whole-job particle-steps/s: all ranks' particles over the slowest rank's time."""
    return npart * steps * world / (ms_max / 1e3)


def reduce_max(pg, value: float, local: int) -> float:
    if pg is None:
        return value
    import torch

    dev = f"cuda:{local}" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


def run_ours(args):
    import mgglam_b200 as m

    world, rank, local, pg = dist_setup(args.gpus)
    w = WORKLOADS[args.workload]
    astep0 = m.astep_for_nsteps(A0, w["nsteps"])
    npart = w["nrow"] ** 3
    seed = replica_seed(w["seed"], rank)
    prec = m.PREC_MIXED if args.precision == "mixed" else m.PREC_PLAIN

    model, mdesc = MODELS[w["model"]]

    def make_box(precision):
        cfg = m.make_config(w["ngrid"], w["nrow"], w["box"], om=COSMO["om"], oml=COSMO["oml"], omb=COSMO["omb"],
                            mg_model=model, fr_n=1, fr0=-1e-5, cycle="V", iter_count_max=4, res_conv=1e-8,
                            precision=precision, device=local)
        b = m.Box(cfg)
        if model in (m.MODEL_KMOUFLAGE, m.MODEL_CSF):
            b.set_background(m.background_table(cfg)[0])
        return b

    def timed_run(box, profile):
        """Steps 1..K of the schedule from the initial conditions at a = 0.02 (the
        untimed warm-up steps ran before on the same box); device ms by CUDA events.
        One mgg_step call (the main-loop body) per step."""
        box.make_ics(seed=seed, aexpn=A0, astep=astep0)
        st = box.new_state(A0, astep0)
        if profile:
            box.profile_reset()
            box.profile(True)
        barrier(pg)
        box.synchronize()
        cycles = 0
        reasons = {}
        with ClockSampler(local) as clk:
            box.timer_start()
            for _ in range(args.steps):
                box.step(st)
                cycles += st.report.cycles
                why = EXIT_REASONS.get(st.report.exit_reason, str(st.report.exit_reason))
                reasons[why] = reasons.get(why, 0) + 1
            ms = box.timer_stop()
        box.synchronize()
        barrier(pg)
        box.profile(False)
        box.set_time(st.aexpn, st.astep)
        pk = box.power(True)
        pos = box.download_particles()[:3]
        return st, ms, cycles, clk, pk, pos, reasons

    box = make_box(prec)
    box.make_ics(seed=seed, aexpn=A0, astep=astep0)
    wst = box.new_state(A0, astep0)
    for _ in range(args.warmup):
        box.step(wst)
    st, ms, cycles, clk, pk, pos, reasons = timed_run(box, True)
    prof = box.profile_read()
    buckets = box.timing()
    box.close()
    ms_max = reduce_max(pg, ms, local)
    value = aggregate_value(npart, args.steps, world, ms_max)
    a_start = A0

    # the plain drop-in path over the same steps, and the P(k) of the timed form against it
    plain = None
    if prec != m.PREC_PLAIN and not args.no_plain_path:
        pbox = make_box(m.PREC_PLAIN)
        pbox.make_ics(seed=seed, aexpn=A0, astep=astep0)
        pst = pbox.new_state(A0, astep0)
        for _ in range(args.warmup):
            pbox.step(pst)
        _, pms, pcycles, _, ppk, ppos, _ = timed_run(pbox, True)
        pbox.close()
        pms_max = reduce_max(pg, pms, local)
        half = w["ngrid"] // 4   # k < k_Nyq / 2: the first NGRID/4 linear bins
        err = np.abs(pk["pk"][:half] / ppk["pk"][:half] - 1.0)
        dmax = 0.0
        for a, b in zip(pos, ppos):
            d = np.abs(a.astype(np.float64) - b.astype(np.float64))
            dmax = max(dmax, float(np.minimum(d, w["ngrid"] - d).max()))
        plain = {"value": aggregate_value(npart, args.steps, world, pms_max), "ms_per_step": pms_max / args.steps,
                 "mg_cycles_timed": pcycles, "speedup_of_timed_form": pms_max / ms_max,
                 "pk_max_rel_err_vs_plain": float(err.max()), "pk_err_at_k_h_mpc": float(pk["k"][int(err.argmax())]),
                 "pk_bins": f"k < k_Nyq/2 ({half} linear bins) at a = {st.aexpn:.4f}",
                 "max_displacement_vs_plain_cells": dmax}
    del pos

    # roofline of the dominant kernel class
    peak, peak_kind = measured_peaks()
    dom = max(prof.items(), key=lambda kv: kv[1]["ms"])
    dname, d = dom
    per_launch_bytes = d["bytes"] / max(d["launches"], 1)
    avg_ms = d["ms"] / max(d["launches"], 1)
    achieved = per_launch_bytes / (avg_ms / 1e3) / 1e9 if avg_ms > 0 else 0.0
    traffic = ncu_traffic(dname, args.workload)
    launches = int(sum(v["launches"] for v in prof.values()))

    # end to end through the C ABI with host buffers: H2D particles, step, D2H particles
    import torch

    box = make_box(prec)
    box.make_ics(seed=seed, aexpn=A0, astep=astep0)
    host = [torch.empty(npart, dtype=torch.float32, pin_memory=True).numpy() for _ in range(6)]
    cur = box.download_particles()
    for h, c in zip(host, cur):
        h[:] = c
    del cur
    import ctypes

    fp = [h.ctypes.data_as(ctypes.POINTER(ctypes.c_float)) for h in host]
    e2e_steps = args.steps
    barrier(pg)
    box.synchronize()
    box.timer_start()
    mst = box.new_state(A0, astep0)
    for _ in range(e2e_steps):
        # one main-loop step through the C ABI with the particles in pinned host memory:
        # H2D of all six arrays, the step, D2H of all six (mgg_step_host_pipelined: the
        # velocity download runs behind the next step's position upload, density, scalar
        # field and potential; the timer stops after the last one)
        box._check(box.lib.mgg_step_host_pipelined(box.h, ctypes.byref(mst), *fp, npart))
    e2e_ms = box.timer_stop()
    box.synchronize()
    e2e_ms_max = reduce_max(pg, e2e_ms, local)
    e2e_value = aggregate_value(npart, e2e_steps, world, e2e_ms_max)
    box.close()

    forms = None
    if world == 1 and not args.no_forms:
        forms = {"batched": run_batched(m, local, precision=m.PREC_MIXED),
                 "batched_plain": run_batched(m, local, precision=m.PREC_PLAIN),
                 "served": run_served(m, local, nreq=args.served_requests, precision=m.PREC_MIXED),
                 "served_plain": run_served(m, local, nreq=args.served_requests, precision=m.PREC_PLAIN),
                 "models": run_models(m, local)}

    if rank != 0:
        if pg is not None:
            pg.destroy_process_group()
        return
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        v, cores, sample, step_ms = run_cpu(steps=10, warmup=1, workload=args.workload)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample,
               "ms_per_step": step_ms}
    line = {
        "metric": metric_of(args.workload), "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": args.workload, "model": mdesc,
                   "nparticles": npart, "ngrid": w["ngrid"], "box_mpc_h": w["box"],
                   "ics": f"Zel'dovich, BBKS sigma8=0.8159, a0={A0}, seed={w['seed']}+rank",
                   "schedule_steps": w["nsteps"], "a_range": [round(a_start, 5), round(st.aexpn, 5)],
                   "mg": "V-cycle, res_conv 1e-8, iter_count_max 4", "mg_cycles_timed": cycles,
                   "mg_exit_reasons_timed": reasons,
                   "l2": "inputs larger than L2 (4 GiB grids)", "parallelism": f"replicas x{world}",
                   "timing": "device time (CUDA events on the context stream) of steps 1..K of the schedule from "
                             "a=0.02 (K=100 runs to z=0; later steps are slower, the density being more clustered); "
                             "per-launch CUDA events are on for the kernel table, which turns off the CUDA-graph "
                             "replay of the multigrid cycles (about 1 % of a step)",
                   "precision": PRECISION_DOC[args.precision]},
        "plain_path": plain,
        "roofline": {"bound": "hbm", "kernel": dname, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                     "alg_bytes_per_launch": per_launch_bytes, "avg_launch_ms": avg_ms},
        # per kernel class: launches, device ms (CUDA events), algorithmic GB/s and
        # its fraction of the measured HBM peak
        "kernels": {k: {"launches": v["launches"], "ms": round(v["ms"], 3),
                        "gbs": (v["bytes"] / (v["ms"] / 1e3) / 1e9 if v["ms"] > 0 else 0.0),
                        "hbm_frac": (v["bytes"] / (v["ms"] / 1e3) / 1e9 / peak if v["ms"] > 0 else 0.0)}
                    for k, v in prof.items() if v["launches"]},
        "buckets_ms": {"force": buckets[1], "move": buckets[2], "density": buckets[3], "mg": buckets[8]},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 24 * npart, "d2h_bytes_per_step": 24 * npart,
                "steps": e2e_steps, "api": "mgg_step_host_pipelined (pinned host arrays; every step uploads all six "
                                           "particle arrays and downloads all six)"},
        "gpu_launches": launches,
        "clocks": clk.summary(),
        "mg_vcycles_per_s": cycles / (ms_max / 1e3),
        "forms": forms,
    }
    print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()


def run_batched(m, device, nbox=64, steps=3, precision=0):
    """Batched form on the many-small-boxes workload: nbox boxes of 64^3 particles
    on 128^3 meshes (L = 128 Mpc/h), f(R) with |fR0| log-uniform in [1e-7, 1e-4] and
    n in {1, 2}, seeds 1..nbox, on the 40-step schedule.  Times `steps` batched steps
    (mgg_step_batch, all boxes concurrently) after two warm-up steps (the eager first
    solve and the first graphed one, which builds the solve's graph), then runs every
    box again alone from the same initial conditions through mgg_step (the same
    2 + steps steps), times its `steps` steps, and compares its particles with the
    batched box's, bit for bit."""
    rng = np.random.default_rng(4)
    astep0 = m.astep_for_nsteps(A0, 40)
    cfgs = []
    for i in range(nbox):
        fr0 = -float(10.0 ** rng.uniform(-7.0, -4.0))
        cfgs.append(m.make_config(128, 64, 128.0, om=COSMO["om"], oml=COSMO["oml"], omb=COSMO["omb"],
                                  mg_model=m.MODEL_FR, fr_n=int(rng.integers(1, 3)), fr0=fr0, cycle="V",
                                  iter_count_max=4, res_conv=1e-8, precision=precision, device=device))

    def make(i):
        b = m.Box(cfgs[i])
        b.make_ics(seed=i + 1, aexpn=A0, astep=astep0)
        return b

    boxes = [make(i) for i in range(nbox)]
    states = [b.new_state(A0, astep0) for b in boxes]
    idx = list(range(nbox))
    # a box whose scalar-field solve stops converging (residual not finite) leaves the
    # batch; it is reported, not counted in the throughput
    diverged = []

    def batch_step():
        bad = m.step_batch(boxes, states, raise_on_error=False)
        for j in sorted(bad, reverse=True):
            i = idx[j]
            diverged.append({"seed": i + 1, "fr_n": int(cfgs[i].fr_n), "fr0": float(cfgs[i].fr0),
                             "step": int(states[j].istep) + 1})
            boxes.pop(j).close()
            states.pop(j)
            idx.pop(j)
        return len(bad)

    for _ in range(2):   # warm-up: the eager first solve, then the first graphed solve (graph built)
        batch_step()
    t0 = time.perf_counter()
    ps = 0
    for _ in range(steps):
        n_before = len(boxes)
        lost = batch_step()
        ps += (n_before - lost) * 64 ** 3
    for b in boxes:
        b.synchronize()
    t_batch = time.perf_counter() - t0
    cycles = int(sum(st.report.cycles for st in states))
    # every box again alone, from the same initial conditions
    t_one, ps1, equal, compared = 0.0, 0, True, 0
    for b, st, i in zip(boxes, states, idx):
        a = make(i)
        sa = a.new_state(A0, astep0)
        try:
            for _ in range(2):
                a.step(sa)
            a.synchronize()
            t1 = time.perf_counter()
            for _ in range(steps):
                a.step(sa)
            a.synchronize()
            t_one += time.perf_counter() - t1
            ps1 += steps * 64 ** 3
            same = all(np.array_equal(x.view(np.uint32), y.view(np.uint32))
                       for x, y in zip(a.download_particles(), b.download_particles()))
            equal = equal and same and sa.ekin == st.ekin
            compared += 1
        except m.MGGError:
            equal = False
        a.close()
    for b in boxes:
        b.close()
    return {"workload": f"{nbox} x (64^3 particles, 128^3 mesh, L=128), f(R) n in {{1,2}}, |fR0| in [1e-7,1e-4], "
                        f"seeds 1..{nbox}, 40-step schedule from a=0.02",
            "value": ps / t_batch, "unit": UNIT, "ms_per_batch_step": 1e3 * t_batch / steps,
            "one_at_a_time": ps1 / t_one if t_one > 0 else None,
            "speedup_vs_one_at_a_time": (ps / t_batch) / (ps1 / t_one) if ps1 else None,
            "equal_to_one_at_a_time": equal, "boxes_compared": compared,
            "mg_cycles_last_step": cycles, "diverged": diverged, "precision": "mixed" if precision else "plain",
            "timing": "host wall clock around device-synchronised steps"}


def run_served(m, device, nreq=40, rate=20.0, budget_gb=60.0, max_active=8, precision=0):
    """Serving form: nreq requests with Poisson arrivals at `rate`/s, NGRID in
    {64,128,256,512} with p = {.4,.3,.2,.1}, NROW = NGRID/2, L = NGRID Mpc/h, the model
    drawn uniformly from f(R) F5 n=1, nDGP (H0rc=1), symmetron (a*=0.5) and k-mouflage
    (n=3, K0=1, beta=0.1), 20-60 steps each from a=0.02 on the 100-step schedule;
    result = P(k) of the final density.  Reports time-to-result p50/p99 and the
    particle-steps/s of the whole run, after an untimed warm-up request per grid
    size and model."""
    rng = np.random.default_rng(5)
    astep0 = m.astep_for_nsteps(A0, 100)
    models = [m.MODEL_FR, m.MODEL_DGP, m.MODEL_SYMMETRON, m.MODEL_KMOUFLAGE]
    # untimed warm-up: one short request per grid size and model (first launches of
    # each kernel, the chunk tuning of each size), then the timed stream on a new server
    warm = m.Server(device=device, hbm_budget_gb=budget_gb, max_active=max_active)
    wids = []
    for ng in (64, 128, 256, 512):
        for model in models:
            cfg = m.make_config(ng, ng // 2, float(ng), om=COSMO["om"], oml=COSMO["oml"], omb=COSMO["omb"],
                                mg_model=model, fr_n=1, fr0=-1e-5, cycle="V", iter_count_max=4, res_conv=1e-8,
                                precision=precision, device=device)
            wids.append((warm.submit(cfg, 1, A0, astep0, 2), ng))
    for rid, ng in wids:
        warm.wait(rid, ng // 2)
    warm.close()
    srv = m.Server(device=device, hbm_budget_gb=budget_gb, max_active=max_active)
    plan = []
    t = 0.0
    for i in range(nreq):
        t += rng.exponential(1.0 / rate)
        ng = int(rng.choice([64, 128, 256, 512], p=[0.4, 0.3, 0.2, 0.1]))
        plan.append((t, ng, int(rng.choice(models)), int(rng.integers(20, 61)), 1000 + i))
    ids = []
    t0 = time.perf_counter()
    for (ta, ng, model, nsteps, seed) in plan:
        dt = ta - (time.perf_counter() - t0)
        if dt > 0:
            time.sleep(dt)
        cfg = m.make_config(ng, ng // 2, float(ng), om=COSMO["om"], oml=COSMO["oml"], omb=COSMO["omb"],
                            mg_model=model, fr_n=1, fr0=-1e-5, cycle="V", iter_count_max=4, res_conv=1e-8,
                            precision=precision, device=device)
        ids.append((srv.submit(cfg, seed, A0, astep0, nsteps), ng, nsteps))
    lat, ps = [], 0
    for rid, ng, nsteps in ids:
        info, _, _, _ = srv.wait(rid, ng // 2)
        lat.append(info.t_done_ms - info.t_submit_ms)
        ps += (ng // 2) ** 3 * nsteps
    makespan = time.perf_counter() - t0
    srv.close()
    lat = np.array(lat)
    return {"workload": f"{nreq} requests, Poisson {rate}/s, NGRID 64-512 (p .4/.3/.2/.1), f(R)/nDGP/symmetron/"
                        "k-mouflage, 20-60 steps, P(k) at the end",
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "value": ps / makespan, "unit": UNIT, "makespan_s": makespan, "requests": nreq,
            "budget_gb": budget_gb, "max_active": max_active, "precision": "mixed" if precision else "plain"}


def run_models(m, device, steps=2):
    """The modified-gravity families on 256^3 particles / 512^3 mesh (L = 512 Mpc/h):
    f(R) F5 n=1, nDGP (H0rc=1, normal branch), symmetron (a*=0.5, beta=1,
    lambda_phi=1 Mpc/h), k-mouflage (n=3, K0=1, beta=0.1) and the coupled scalar
    field (alpha=0.1, beta=-0.2), from a=0.6 (all solvers active), V-cycles,
    iter_count_max 4.  Device time per step (CUDA events) after one warm-up step,
    on the plain path and in the precision form from the same initial conditions,
    with the largest relative P(k) difference between the two (k < k_Nyq/2)."""
    out = {}
    for name, model in (("f(R)", m.MODEL_FR), ("nDGP", m.MODEL_DGP), ("symmetron", m.MODEL_SYMMETRON),
                        ("k-mouflage", m.MODEL_KMOUFLAGE), ("csf", m.MODEL_CSF)):
        res, pks = {}, {}
        for form, prec in (("plain", m.PREC_PLAIN), ("mixed", m.PREC_MIXED)):
            cfg = m.make_config(512, 256, 512.0, om=COSMO["om"], oml=COSMO["oml"], omb=COSMO["omb"], mg_model=model,
                                cycle="V", iter_count_max=4, res_conv=1e-8, precision=prec, device=device)
            tab = None
            if model in (m.MODEL_KMOUFLAGE, m.MODEL_CSF):
                tab, _ = m.background_table(cfg)
            b = m.Box(cfg)
            if tab is not None:
                b.set_background(tab)
            b.make_ics(seed=11, aexpn=0.6, astep=0.01)
            st = b.new_state(0.6, 0.01)
            b.step(st)
            b.timer_start()
            cycles = 0
            for _ in range(steps):
                b.step(st)
                cycles += st.report.cycles
            ms = b.timer_stop() / steps
            b.set_time(st.aexpn, st.astep)
            pks[form] = b.power(True)["pk"]
            b.close()
            res[form] = {"ms_per_step": ms, "value": 256 ** 3 / (ms / 1e3), "mg_cycles_per_step": cycles / steps}
        err = np.abs(pks["mixed"][:128] / pks["plain"][:128] - 1.0)
        out[name] = {"ms_per_step": res["plain"]["ms_per_step"], "value": res["plain"]["value"], "unit": UNIT,
                     "mg_cycles_per_step": res["plain"]["mg_cycles_per_step"],
                     "precision_form": dict(res["mixed"], speedup=res["plain"]["ms_per_step"] / res["mixed"]["ms_per_step"],
                                            pk_max_rel_err_vs_plain=float(err.max()))}
    return out


def run_cpu_full(workload: str, steps: int = 1):
    """The oracle port on all host threads on the workload itself: numpy Zel'dovich
    initial conditions of the workload's particles, mesh, box and seed at a = 0.02,
    then steps 1..steps of its schedule.  Returns (particle-steps/s, cores, sample,
    ms per step, seconds spent on the initial conditions)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import mgglam_b200 as m
    import oracle as orc

    w = WORKLOADS[workload]
    model, mdesc = MODELS[w["model"]]
    nt = os.cpu_count() or 1
    astep0 = m.astep_for_nsteps(A0, w["nsteps"])
    cfg = m.make_config(w["ngrid"], w["nrow"], w["box"], om=COSMO["om"], oml=COSMO["oml"], omb=COSMO["omb"],
                        mg_model=model, fr_n=1, fr0=-1e-5, cycle="V", iter_count_max=4, res_conv=1e-8)
    bg = m.background_table(cfg)[0] if model in (m.MODEL_KMOUFLAGE, m.MODEL_CSF) else None
    t0 = time.perf_counter()
    parts = numpy_ics(w["nrow"], w["ngrid"], w["box"], w["seed"], A0, astep0)
    t_ics = time.perf_counter() - t0
    st = {"a": A0, "da": astep0, "sf": float(np.float32(np.float32(astep0) / np.float32(A0)))}
    fi2 = np.zeros(w["ngrid"] ** 3, np.float32)
    t0 = time.perf_counter()
    for i in range(1, steps + 1):
        fi2, parts = cpu_step(orc, cfg, st, fi2, parts, i, nt, bg)
    dt = time.perf_counter() - t0
    sample = (f"steps 1..{steps} of the workload itself ({w['nrow']}^3 particles, {w['ngrid']}^3 mesh, "
              f"L = {w['box']:g} Mpc/h, {mdesc}, {w['nsteps']}-step schedule from a={A0}), from numpy Zel'dovich "
              f"initial conditions of seed {w['seed']}; C++/OpenMP restatement of the reference, {nt} threads")
    return w["nrow"] ** 3 * steps / dt, nt, sample, dt / steps * 1e3, t_ics


def run_reference(args):
    """The reference arm: the CPU restatement of the reference's path on the host
    cores, on the same workload as the GPU arm.  One step of the workload is a
    couple of minutes of host work at 512^3 / 1024^3, so the arm times
    --ref-steps full-size steps (default 1: step 1 of the schedule) whatever
    --steps is, after --warmup steps of the 128^3 / 256^3 sample of the same
    model and cell size (which load the library and page in the host memory)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if args.warmup > 0:
        run_cpu(steps=1, warmup=max(args.warmup - 1, 0), workload=args.workload)
    value, cores, sample, step_ms, t_ics = run_cpu_full(args.workload, steps=max(1, args.ref_steps))
    w = WORKLOADS[args.workload]
    line = {
        "metric": metric_of(args.workload), "value": value, "unit": UNIT, "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": max(1, args.ref_steps), "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": args.workload, "nparticles": w["nrow"] ** 3, "ngrid": w["ngrid"], "box_mpc_h": w["box"],
                   "same_config": True, "ics_seconds": t_ics},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="fr5_512_1024")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the batched and served forms")
    ap.add_argument("--ref-steps", type=int, default=1,
                    help="full-size steps the reference arm times (each takes minutes on the host cores)")
    ap.add_argument("--served-requests", type=int, default=40,
                    help="requests of the served stream (the full served workload is 2000)")
    ap.add_argument("--precision", choices=["mixed", "plain"], default="mixed",
                    help="the timed form; with mixed the plain path is also timed over the same steps")
    ap.add_argument("--no-plain-path", action="store_true",
                    help="do not time the plain path beside the precision form (profiling runs)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
