#!/usr/bin/env python
"""Benchmark of the VMC hot path (RBM + pair-product wavefunction, J1-J2 Heisenberg model).

One step = one stochastic-reconfiguration iteration of main.f90:311-453 over all walkers:
update_slater_elements, make_sample (warm-up + stored sweeps), the estimators of
calc_phys_quantity_opt, the S = O^T O build, the Cholesky solve that replaces pdposv, and the
parameter update.  The metric is MC samples/s (stored samples per second; SR steps/s reported
beside it) on the 10x10 periodic lattice at J2/J1 = 0.5 with a translation-symmetric RBM
(alpha = 4, 100 projections, so 200 Pfaffian blocks per walker), 4096 walkers, 65536 samples per
SR step.  Synthetic seeded inputs with the reference's shapes stand in for its input files.

Usage:  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
        [--workload NAME] [--precision fp64|split]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MC samples/s and SR steps/s at 10x10 J2=0.5, chosen vs plain FP64, dE/site"
# DRAM bytes (read + write) that ncu counted for one sampler_stream_kernel launch of the 1-wave 10x10
# workload (one walker per SM, one stored sample), divided by that launch's algorithmic bytes
SAMPLER_TRAFFIC_PER_ALG_BYTE = (2.0793e12 + 0.6517e12) / 3.1765e12
# wall-clock budget of one bench process: the plain all-FP64 twin trajectory gets as many of the K steps as fit
PAIR_BUDGET_S = 1450.0
T_START = time.perf_counter()

WORKLOADS = {
    # 10x10 at scale: translation-symmetric RBM (alpha=4, 100 projections), 4096 walkers, 65536 samples per step
    "j1j2_10x10_trans": dict(L=10, translations=True, alphar=4, orbital="full", walkers=4096, ns=16, J2=0.5),
    # same lattice without translation projection (2 Pfaffian blocks per walker)
    "j1j2_10x10_single": dict(L=10, translations=False, alphar=4, orbital="full", walkers=4096, ns=16, J2=0.5),
    "j1j2_6x6_trans_small": dict(L=6, translations=True, alphar=2, orbital="full", walkers=256, ns=16, J2=0.5),
    # 10x10 without translation projection, 16384 samples: a few-GB profiling case of the S build (Nv = 10404)
    "j1j2_10x10_single_16k": dict(L=10, translations=False, alphar=4, orbital="full", walkers=1024, ns=16, J2=0.5),
    # one wave of walkers (one per SM), one stored sample each: the profiling case of the 10x10 kernels
    "j1j2_10x10_trans_1wave": dict(L=10, translations=True, alphar=4, orbital="full", walkers=148, ns=1, J2=0.5),
    # correlation measurement (the Calc_Correlation program) of 16384 samples on the 10x10 translation-symmetric state
    "corr_10x10_trans": dict(L=10, translations=True, alphar=4, orbital="full", walkers=4096, ns=4, J2=0.5),
}


def _rank_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(
        os.environ.get("LOCAL_RANK", "0"))


def make_problem(w, seed=2024):
    from rbm_pp_b200 import formats as fm
    return fm.synthetic_problem(w["L"], translations=w["translations"], alphar=w["alphar"], orbital=w["orbital"],
                                nsample=w["walkers"] * w["ns"], seed=seed, J2=w["J2"])


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def cpu_baseline(w, problem, max_threads=None):
    """The oracle (a line-by-line CPU restatement of the reference's make_sample and calc_phys_quantity_opt)
    on the host cores, one walker per thread, each walker a complete make_sample of the workload (warm-up plus
    every stored sweep) and the measurement of all its samples.  The rate (stored samples per second) needs no
    extrapolation; only the time of a whole step is scaled by the walker count."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    cores = os.cpu_count() or 1
    threads = min(cores, max_threads or 64, po.max_threads() if po.max_threads() > 0 else cores)
    walkers, ns = w["walkers"], w["ns"]
    o = po.Oracle(problem, nranks=threads, nsample_per_rank=ns, nthreads=threads)
    o.set_params(problem.br, problem.Wr, problem.slater, 0.0)
    o.seed(777)
    t0 = time.perf_counter()
    o.make_sample(True)
    t1 = time.perf_counter()
    m = o.measure(want_S=False)
    t2 = time.perf_counter()
    t_sample = t2 - t0
    return {"value": threads * ns / t_sample, "unit": "MC samples/s", "cores": threads, "kind": "port",
            "sample": (f"oracle make_sample ({max(30, ns // 100)} + {ns} sweeps) and measure of {threads} walkers x "
                       f"{ns} stored samples, one walker per thread, in {t_sample:.1f} s (sampling {t1 - t0:.1f} s, "
                       f"measurement {t2 - t1:.1f} s); a {walkers}-walker step would take "
                       f"{t_sample * walkers / threads:.0f} s"),
            "measured_s": t_sample, "step_s_extrapolated": t_sample * walkers / threads,
            "energy_per_site": m["Etot"] / m["norm"] / (w["L"] ** 2)}


def run_reference(args):
    """The reference arm: the oracle port on the host cores, each step one complete sample of the workload
    (threads walkers, full make_sample + measurement); warm-up is one such step (the CPU has nothing to warm
    beyond that)."""
    rank, world, _ = _rank_env()
    if rank != 0:
        return 0
    w = WORKLOADS[args.workload]
    problem = make_problem(w)
    for _ in range(min(args.warmup, 1)):
        cpu_baseline(w, problem)
    vals, meas = [], []
    info = None
    for _ in range(args.steps):
        info = cpu_baseline(w, problem)
        vals.append(info["value"])
        meas.append(info["measured_s"])
    v = float(np.median(vals))
    ms = w["walkers"] * w["ns"] / v * 1e3
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "MC samples/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": min(args.warmup, 1), "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "L": w["L"], "walkers": w["walkers"],
                       "samples_per_step": w["walkers"] * w["ns"], "alphar": w["alphar"],
                       "n_mp_trans": w["L"] ** 2 if w["translations"] else 1, "J2": w["J2"]},
            "measured_s_per_step": meas,
            "ms_per_step_basis": "the measured complete walkers, scaled by walker count to the full step",
            "cpu_baseline": {k: info[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": v, "unit": "MC samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


BATCH_LS = (12, 14, 16, 18)
BATCH_J2 = (0.40, 0.45, 0.50, 0.55, 0.60)


def run_batch(args):
    """Batched sampling over lattices L = 12..18 crossed with J2/J1 = 0.40..0.60 (1024 walkers each,
    alpha = 2, no translation projection, N_QP = 2): one persistent launch per make_sample, launch shape
    and walker order picked by the autotuner.  Reports aggregate MC samples/s of the batched launch and,
    for comparison, each instance's MC samples/s when launched alone."""
    import torch
    from rbm_pp_b200 import capi
    from rbm_pp_b200 import formats as fm
    torch.cuda.set_device(0)
    walkers, ns = (1024, 4) if args.workload == "batch_l12_18" else (64, 2)
    ctxs, meta = [], []
    for L in BATCH_LS:
        for J2 in BATCH_J2:
            p = fm.synthetic_problem(L, translations=False, alphar=2, orbital="full", nsample=walkers * ns,
                                     seed=100 + L, J2=J2)
            g = capi.Context(p, n_walkers=walkers, nsample_per_walker=ns)
            g.set_params(p.br, p.Wr, p.slater, 0.0)
            g.seed(4000 + 10 * L + int(100 * J2))
            ctxs.append(g)
            meta.append((L, J2))
    b = capi.Batch(ctxs)
    threads, order, probe_ms = b.tune()
    b.make_sample(True)
    for _ in range(max(0, args.warmup - 1)):
        b.make_sample(False)
    clk = ClockSampler(0)
    clk.start()
    ms = []
    for _ in range(args.steps):
        b.make_sample(False)
        ms.append(ctxs[0].stats()["sampler_ms"])
    clocks = clk.stop()
    batch_ms = float(np.mean(ms))
    total_samples = walkers * ns * len(ctxs)
    # each instance alone (same direct sampler), one make_sample each
    os.environ["RBMPP_SAMPLER"] = "direct"
    alone = []
    for g, (L, J2) in zip(ctxs, meta):
        g.make_sample(False)
        t = g.stats()["sampler_ms"]
        alone.append({"L": L, "J2": J2, "ms": t, "samples_per_s": walkers * ns / (t * 1e-3)})
    os.environ.pop("RBMPP_SAMPLER", None)
    line = {"metric": "MC samples/s, batched lattices L=12..18 x J2/J1=0.40..0.60 in one launch",
            "value": total_samples / (batch_ms * 1e-3), "unit": "MC samples/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": batch_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, reference file shapes)",
            "config": {"workload": args.workload, "instances": len(ctxs), "walkers_per_instance": walkers,
                       "samples_per_walker": ns, "alphar": 2, "n_qp": 2,
                       "tuned": {"threads": threads, "order": ["context-major", "round-robin",
                                                                "longest-first"][order],
                                 "probe_ms": probe_ms}},
            "unbatched_sum_ms": float(sum(a["ms"] for a in alone)),
            "per_instance_alone": alone, "clocks": clocks}
    print(json.dumps(line), flush=True)
    b.close()
    for g in ctxs:
        g.close()
    return 0


def corr_flops_per_sample(w):
    """Algorithmic FP64 flops of one correlation-measured sample, per projection: the scratch inverse
    (2 Np^3), one mat-vec W = Y v per up electron (2 Np^3) and two dot products of length Np per
    up-down pair (4 Np^3)."""
    np_ = w["L"] ** 2 // 2
    n_qp = 2 * (w["L"] ** 2 if w["translations"] else 1)
    return n_qp * 8.0 * np_ ** 3


def run_corr(args):
    """The correlation measurement of the Calc_Correlation program (Chi_sp for every site pair, Chi_vbs
    per bond type, energy scalars) on the stored samples of one make_sample, through the C ABI."""
    import torch
    from rbm_pp_b200 import capi
    torch.cuda.set_device(0)
    w = WORKLOADS[args.workload]
    problem = make_problem(w)
    g = capi.Context(problem, n_walkers=w["walkers"], nsample_per_walker=w["ns"])
    g.set_params(problem.br, problem.Wr, problem.slater, 0.0)
    g.seed(2024)
    g.make_sample(True)
    launches0 = g.kernel_launches()
    for _ in range(args.warmup):
        g.measure_correlation()
    clk = ClockSampler(0)
    clk.start()
    kern, wall = [], []
    launches0 = g.kernel_launches()
    for _ in range(args.steps):
        t0 = time.perf_counter()
        m = g.measure_correlation()
        wall.append(time.perf_counter() - t0)
        kern.append(g.stats()["estimator_ms"])
    clocks = clk.stop()
    launches = g.kernel_launches() - launches0
    n = w["walkers"] * w["ns"]
    wall_s = float(np.mean(wall))
    kern_ms = float(np.mean(kern))
    flops = corr_flops_per_sample(w) * n
    achieved = flops / (kern_ms * 1e-3) / 1e12
    nchi = w["L"] ** 2 * (w["L"] ** 2 + 1) // 2
    line = {"metric": "correlation-measured samples/s at 10x10 J2=0.5 (Chi_sp over all site pairs, Chi_vbs)",
            "value": n / wall_s, "unit": "samples/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": wall_s * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded, reference file shapes)",
            "config": {"workload": args.workload, "L": w["L"], "walkers": w["walkers"], "samples_per_step": n,
                       "alphar": w["alphar"], "n_qp": 2 * (w["L"] ** 2 if w["translations"] else 1),
                       "l2": "per-sample rows larger than L2"},
            "kernel_ms": kern_ms,
            "roofline": {"kernel": "correlation_kernel", "bound": "fp64", "achieved": achieved, "peak": 40.0,
                         "unit": "TFLOP/s", "frac": achieved / 40.0,
                         "peak_kind": "nominal FP64 (no measured FP64 peak on this pool)", "traffic": None,
                         "algorithmic_flops": flops},
            "energy_per_site": m["Etot"] / m["norm"] / w["L"] ** 2, "clocks": clocks, "gpu_launches": launches,
            "e2e": {"value": n / wall_s, "unit": "samples/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 8 * (5 + 6 * nchi)}}
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle as po
        cores = os.cpu_count() or 1
        threads = min(cores, 64, po.max_threads() if po.max_threads() > 0 else cores)
        o = po.Oracle(problem, nranks=threads, nsample_per_rank=1, nthreads=threads)
        o.set_params(problem.br, problem.Wr, problem.slater, 0.0)
        o.seed(777)
        o.make_sample(True)
        t0 = time.perf_counter()
        o.measure_correlation()
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": threads / dt, "unit": "samples/s", "cores": threads, "kind": "port",
                                "sample": f"oracle correlation measurement of {threads} samples (one per thread) "
                                          f"in {dt:.1f} s"}
    print(json.dumps(line), flush=True)
    g.close()
    return 0


def run_ours(args):
    import torch
    rank, world, local = _rank_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from rbm_pp_b200 import capi
    from rbm_pp_b200 import distributed as rdist
    w = WORKLOADS[args.workload]
    problem = make_problem(w)
    prec = capi.SR_SPLIT_BF16 if args.precision == "split" else capi.SR_FP64
    ctx = capi.Context(problem, n_walkers=w["walkers"], nsample_per_walker=w["ns"], device=local,
                       walker_offset=rank * w["walkers"])
    runner = rdist.SRRunner(ctx, problem, iseed0=12345, precision=prec, world=world, rank=rank)
    for _ in range(args.warmup):
        runner.step()
    torch.cuda.synchronize()
    # the plain all-FP64 twin continues from the same state (walkers, streams, parameters, bookkeeping)
    twin = None
    if world == 1 and args.precision == "split" and not args.no_plain:
        twin = capi.Context(problem, n_walkers=w["walkers"], nsample_per_walker=w["ns"], device=local,
                            walker_offset=0)
        twin.copy_state_from(ctx)
    if world > 1:
        torch.distributed.barrier()
    clk = ClockSampler(torch.cuda.current_device())
    clk.start()
    step_ms, samp_ms, est_ms, sb_ms, solve_ms, ref_ms, acc_all, props, energies = [], [], [], [], [], [], [], [], []
    refine, e2e_ms = [], []
    launches0 = ctx.kernel_launches()
    br, Wr, sl, sh = ctx.get_params()
    h2d = d2h = br.nbytes + Wr.nbytes + sl.nbytes + 8
    for _ in range(args.steps):
        # end to end through the public API: the step's parameters in from host buffers, its energy and the new
        # parameters back to the host; the device time of the same step is `value`'s
        t0 = time.perf_counter()
        ctx.set_params(br, Wr, sl, sh)
        rec = runner.step()
        br, Wr, sl, sh = ctx.get_params()
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
        st = ctx.stats()
        step_ms.append(rec["device_ms"])
        samp_ms.append(st["sampler_ms"])
        est_ms.append(st["estimator_ms"])
        sb_ms.append(st["sbuild_ms"])
        solve_ms.append(st["solve_ms"])
        ref_ms.append(st["refine_ms"])
        acc_all.append(st["accepts_all"])
        props.append(st["proposals"])
        energies.append(rec["Etot"])
        refine.append((rec.get("refine_iterations", 0), rec.get("refine_residual", 0.0), st["cholesky_attempts"]))
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clocks = clk.stop()
    launches = ctx.kernel_launches() - launches0
    # max over ranks of the device time per step
    t = torch.tensor([float(np.mean(step_ms))], device="cuda")
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ms = float(t.item())
    samples_per_step = w["walkers"] * w["ns"] * world
    value = samples_per_step / (ms * 1e-3)
    e2e_v = samples_per_step / (float(np.mean(e2e_ms)) * 1e-3)
    # the twin: the same steps with the plain all-FP64 S build and Cholesky solve, as many as the budget allows
    plain = None
    if twin is not None:
        left = PAIR_BUDGET_S - (time.perf_counter() - T_START) - (120.0 if not args.no_cpu_baseline else 0.0)
        n_pair = int(max(1, min(args.steps, left // (ms * 1.05e-3))))
        trunner = rdist.SRRunner.attach(twin, problem, capi.SR_FP64)
        pe, pms, psr = [], [], []
        for _ in range(n_pair):
            prec_rec = trunner.step()
            stp = twin.stats()
            pe.append(prec_rec["Etot"])
            pms.append(prec_rec["device_ms"])
            psr.append(stp["sbuild_ms"] + stp["solve_ms"] + stp["refine_ms"])
        chosen_sr = [a + b + c for a, b, c in zip(sb_ms, solve_ms, ref_ms)]
        de = [abs(a - b) / (w["L"] ** 2) for a, b in zip(energies, pe)]
        plain = {"paired_steps": n_pair, "ms_per_step": float(np.mean(pms)),
                 "sr_steps_per_s": 1e3 / float(np.mean(pms)),
                 "energy_per_site": [e / (w["L"] ** 2) for e in pe],
                 "sr_phase_ms": float(np.mean(psr)),
                 "sr_phase_speedup_chosen_vs_plain": float(np.mean(psr)) / float(np.mean(chosen_sr[:n_pair])),
                 "delta_e_per_site": {"per_step": de, "max": float(max(de)), "mean": float(np.mean(de)),
                                      "of_the_mean": abs(float(np.mean(energies[:n_pair])) - float(np.mean(pe)))
                                      / (w["L"] ** 2)}}
        twin.close()
    peaks, peak_kind = measured_peaks()
    Np = (w["L"] ** 2) // 2
    n_qp = 2 * (w["L"] ** 2 if w["translations"] else 1)
    bytes_prop = n_qp * 8.0 * Np * Np
    bytes_acc = n_qp * 16.0 * Np * Np
    alg_bytes = float(np.mean(props)) * bytes_prop + float(np.mean(acc_all)) * bytes_acc
    smp = float(np.mean(samp_ms))
    achieved = alg_bytes / (smp * 1e-3) / 1e9
    line = {"metric": METRIC, "value": value, "unit": "MC samples/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, reference file shapes)",
            "config": {"workload": args.workload, "L": w["L"], "walkers_per_gpu": w["walkers"],
                       "samples_per_step": samples_per_step, "alphar": w["alphar"], "n_qp": n_qp,
                       "n_slater": problem.n_slater, "Nv": ctx.Nv, "J2": w["J2"], "sr_precision": args.precision,
                       "l2": "inputs larger than L2 (Y %.1f GB, O %.1f GB per GPU)" % (
                           w["walkers"] * n_qp * Np * Np * 8 / 1e9, samples_per_step / world * ctx.Nv * 8 / 1e9)},
            "sr_steps_per_s": 1e3 / ms,
            "energy_per_site": [e / (w["L"] ** 2) for e in energies],
            "phases_ms": {"make_sample": smp, "estimator": float(np.mean(est_ms)), "s_build": float(np.mean(sb_ms)),
                          "cholesky_solve": float(np.mean(solve_ms)), "refinement": float(np.mean(ref_ms)),
                          "sr_phase": float(np.mean(sb_ms)) + float(np.mean(solve_ms)) + float(np.mean(ref_ms))},
            "roofline": {"kernel": "sampler_stream_kernel (make_sample)", "bound": "hbm", "achieved": achieved,
                         "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
                         "peak_kind": peak_kind + " (burst copy)",
                         "traffic": (alg_bytes * SAMPLER_TRAFFIC_PER_ALG_BYTE if SAMPLER_TRAFFIC_PER_ALG_BYTE
                                     else None),
                         "traffic_source": "ncu dram bytes / algorithmic bytes of the 1-wave capture, scaled",
                         "algorithmic_bytes": alg_bytes},
            "clocks": clocks,
            "e2e": {"value": e2e_v, "unit": "MC samples/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "sr_refinement": {"iterations": [r[0] for r in refine], "residual": [r[1] for r in refine],
                              "cholesky_attempts": [r[2] for r in refine]},
            "plain_fp64": plain}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline(w, problem)
        line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def run_sr_precision(args):
    """Error table of the split-BF16 SR path at full size (10x10, 100 translations, 4096 walkers x 16 samples,
    Nv = 10404): after W optimisation steps, two contexts in the same state sample identical chains; one builds
    S in FP64, the other in split-BF16 on the tensor cores; both take the SR step (FP64 Cholesky solve, and
    the split one refined on the exact S); then both sample and measure the energy at their new parameters.
    Reported: the S entry error, the SR-direction and lambda errors, the energy-per-site difference, and the
    phase times of both paths."""
    import torch
    from rbm_pp_b200 import capi
    from rbm_pp_b200 import distributed as rdist
    torch.cuda.set_device(0)
    w = WORKLOADS["j1j2_10x10_trans"]
    problem = make_problem(w)
    inp = problem.inp
    a = capi.Context(problem, n_walkers=w["walkers"], nsample_per_walker=w["ns"])
    runner = rdist.SRRunner(a, problem, iseed0=12345, precision=capi.SR_FP64)
    for _ in range(args.warmup):
        runner.step()
    b = capi.Context(problem, n_walkers=w["walkers"], nsample_per_walker=w["ns"])
    b.copy_state_from(a)
    res = {}
    for c, prec, key in ((a, capi.SR_FP64, "fp64"), (b, capi.SR_SPLIT_BF16, "split")):
        c.make_sample(False)
        c.set_s_precision(prec)
        m = c.measure(want_S=True)
        res[key] = dict(m=m, x=c.samples()[0], sbuild_ms=c.stats()["sbuild_ms"])
    assert np.array_equal(res["fp64"]["x"], res["split"]["x"]), "the two contexts sampled different chains"
    m64, m16 = res["fp64"]["m"], res["split"]["m"]
    norm = m64["norm"]
    mv = m64["Ovec"] / norm
    S64 = m64["S"] / norm - np.outer(mv, mv)
    d = m16["S"] / norm - np.outer(mv, mv) - S64
    smax = float(np.abs(S64).max())
    dg = np.diag(S64)
    sd = float(dg[dg > 0].mean())
    table = {"S_max_abs_err_over_max_S": float(np.abs(d).max()) / smax,
             "S_rms_err_over_max_S": float(np.sqrt(np.mean(d * d))) / smax,
             "S_max_abs_err_over_mean_diag": float(np.abs(d).max()) / sd,
             "S_diag_max_rel_err": float(np.abs(np.diag(d)).max() / np.abs(dg).max())}
    del d, S64, m64["S"], m16["S"]
    out = {}
    for c, prec, key in ((a, capi.SR_FP64, "fp64"), (b, capi.SR_SPLIT_BF16, "split")):
        sout, dx = c.sr_step(1000 + args.warmup, inp.delta_tau, inp.s_factor0, inp.s_cut, precision=prec,
                             refine_steps=200)
        st = c.stats()
        out[key] = dict(dx=dx, lam=sout.lambda_, it=sout.refine_iterations, res=sout.refine_residual,
                        attempts=st["cholesky_attempts"], sbuild_ms=res[key]["sbuild_ms"], solve_ms=st["solve_ms"],
                        refine_ms=st["refine_ms"], precond_shift=sout.precond_shift)
    dx64, dx16 = out["fp64"]["dx"], out["split"]["dx"]
    table["dtheta_max_rel_err"] = float(np.abs(dx16 - dx64).max() / np.abs(dx64).max())
    table["lambda_rel_err"] = abs(out["split"]["lam"] - out["fp64"]["lam"]) / abs(out["fp64"]["lam"])
    pa, pb = a.get_params(), b.get_params()
    table["params_max_rel_diff"] = float(max(np.abs(pa[i] - pb[i]).max() / max(np.abs(pa[i]).max(), 1e-300)
                                             for i in range(3)))
    e = {}
    for c, key in ((a, "fp64"), (b, "split")):
        c.make_sample(False)
        me = c.measure_energy()
        e[key] = me["Etot"] / me["norm"] / (w["L"] ** 2)
    table["energy_per_site_fp64"] = e["fp64"]
    table["energy_per_site_split"] = e["split"]
    table["delta_energy_per_site"] = abs(e["split"] - e["fp64"])
    table["next_chains_identical"] = bool(np.array_equal(a.samples()[0], b.samples()[0]))
    sr = {k: {kk: vv for kk, vv in v.items() if kk != "dx"} for k, v in out.items()}
    for k in sr:
        sr[k]["sr_phase_ms"] = sr[k]["sbuild_ms"] + sr[k]["solve_ms"] + sr[k]["refine_ms"]
    line = {"metric": "split-BF16 SR error table and phase times at 10x10 (Nv = 10404, 65536 samples)",
            "value": table["delta_energy_per_site"], "unit": "|dE/site|", "n_gpus": 1, "steps": 1,
            "warmup": args.warmup, "higher_is_better": False, "dtype": "f64 / split-bf16",
            "data": "synthetic (seeded, reference file shapes)",
            "config": {"workload": "sr_precision_10x10", "L": 10, "Nv": a.Nv, "samples": w["walkers"] * w["ns"],
                       "shift": "mean(diag S) * max(1e-4, s_factor0) (SR_pdposv.f90:167-170)"},
            "errors": table, "sr": sr,
            "sr_phase_speedup_chosen_vs_plain": sr["fp64"]["sr_phase_ms"] / sr["split"]["sr_phase_ms"]}
    print(json.dumps(line), flush=True)
    a.close()
    b.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="j1j2_10x10_trans",
                    choices=sorted(WORKLOADS) + ["batch_l12_18", "batch_l12_18_small", "sr_precision_10x10"])
    ap.add_argument("--precision", default="split", choices=["fp64", "split"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the extra all-FP64 comparison step")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload.startswith("batch_"):
        return run_batch(args)
    if args.workload.startswith("corr_"):
        return run_corr(args)
    if args.workload == "sr_precision_10x10":
        return run_sr_precision(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
