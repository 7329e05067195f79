#!/usr/bin/env python
"""Benchmark of the metadynamics hot path: CV + bias + force atom-steps/s.

Workload (the config the headline metric is quoted on): 256,000 atoms in
z-stacked FCC / BCC / hard-core-liquid slabs, STEINH L Q4 + Q6 (STEP
switching at 3.9 A; the cap of 18 is parsed and reported as non-binding),
MEAN_SOLID of each as v1, v2, a 200 x 200 well-tempered grid on [0,1]^2
(TEMP 300, biasf 9 -> delta T = 2400 K), sigma 0.01, h 0.005 eV, PACE 10,
mixed precision (FP32 per atom, FP64 sums and grid).  Positions are seeded
synthetic data: four jittered copies (N(0, 0.05 A)) of the slab geometry,
cycled step by step.

A step = one FixMetadynamics::post_force: cell list, neighbour lists, Q4/Q6
values, reductions, bias grid (deposit every PACE), dV/ds, analytic forces.
`value` times the device-resident call (inputs in HBM); `e2e` times the C-ABI
call on pinned host x and f, H2D and D2H copies included.  L2 is flushed
(a 256 MB write) before every timed step, outside the timed interval.

--impl reference times the reference algorithm's CPU restatement (the FP64
oracle, OpenMP over all host cores) on the same workload; the reference
plugin itself needs LAMMPS, which is absent.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(ROOT, "metad-toy_b200")]

METRIC = "CV+bias+force atom-steps/s at 256k atoms; NN vs exact hill bias, same error"
UNIT = "atom-steps/s"
WORKLOAD = "256k-atom FCC/BCC/liquid slabs, STEINH L Q4+Q6 MEAN_SOLID with forces, 2D 200x200 WT grid, PACE 10"
# neighbour lists: candidates within cutoff + 1.0 A kept across steps, filtered
# to the exact lists every step, rebuilt when an atom moves more than 0.5 A and
# at least every 10 steps (the timed steps include those rebuilds)
SKIN, EVERY = 1.0, 10


def fix_args(skin=SKIN, every=EVERY):
    a = ["GAUSSIAN", 0.01, 0.005, 9.0, "PACE", 10, "TEMP", 300.0,
         "CAL", "NAME", "ST", "SW_FUNC", "STEP", "r_0", 3.9,
         "CAL", "NAME", "Q4", "STEINH", "L", 4, "all", "cutoff_r", 3.9, "cutoff_Natoms", 18, "SW_FUNC_r", "ST",
         "CAL", "NAME", "Q6", "STEINH", "L", 6, "all", "cutoff_r", 3.9, "cutoff_Natoms", 18, "SW_FUNC_r", "ST",
         "SYMBOL", "v1", "Q4.MEAN_SOLID", "SYMBOL", "v2", "Q6.MEAN_SOLID",
         "CV_dim", 2, "DIM", 1, 0, 1, 200, "v1", "DIM", 2, 0, 1, 200, "v2", "WT", 1]
    if skin > 0:
        a += ["NEIGH_SKIN", skin, "NEIGH_EVERY", every]
    return a


def load_base(seed=2024):
    """The slab geometry before jitter (cached: its hard-core liquid takes seconds)."""
    import systems
    cache = os.path.join(tempfile.gettempdir(), "mtd_config2_%d.npz" % seed)
    if os.path.exists(cache):
        z = np.load(cache)
        return z["x"], z["L"]
    x, L = systems.config2(seed=seed)
    np.savez(cache, x=x, L=L)
    return x, L


def load_system(seed=2024, copies=4):
    import systems
    x, L = load_base(seed)
    xs = [np.ascontiguousarray(systems.wrap(systems.jitter(x, 0.05, seed + 1, c), L)) for c in range(copies)]
    return xs, L


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), "mtd_clocks_%d.csv" % os.getpid())

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in open(self.path):
            p = [t.strip() for t in line.split(",")]
            if len(p) >= 7:
                rows.append(p)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = [names[k] for k in range(4) if any(r[3 + k].lower().startswith("active") for r in rows)]
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def kernel_bytes(name, n, nbar):
    """Algorithmic (compulsory) HBM bytes per launch of each kernel of the step
    for STEINH L Q4+Q6 in mixed precision (records of 24 FP32 = 96 B): every
    per-atom array the kernel must read or write once, 4-byte neighbour indices."""
    per_atom = {
        "cell_bin": 32,                       # x 24 -> cell 4, slot 4
        "cell_scatter": 12,                   # cell, slot -> perm
        "cell_sort": 80,                      # perm, x, mask -> xs 24, pf 16, smask, perm
        "neighbors": 24 + 4 * nbar,           # pf 16, cell starts ~4, count 4, indices
        "local_q": 120 + 4 * nbar,            # pf 16, count, indices -> q 96, NF 4
        "local_lq": 228 + 4 * nbar,           # q 96, NF, mask, count, indices -> LQ 96, |LQ| 8, e1/e2 16
        "local_lambda": 216 + 4 * nbar,       # e1/e2 16, LQ 96, NF, count, indices -> lambda 96
        "local_force": 168 + 4 * nbar,        # lambda 96, pf 16, count, indices, perm, f_in 24 -> f_out 24
    }
    return per_atom.get(name, 0.0) * n


def pipeline_bytes(nbar):
    """Compulsory DRAM bytes per atom-step of the whole dependency-minimal
    pipeline (x repack, four passes over positions and lists, q/LQ/adjoint
    records written and read, force read-modify-write): 1070 + 16 nbar."""
    return 1070.0 + 16.0 * nbar


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        p = json.load(open(path))
        return p.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "ncu_dram_per_launch.json")
    if not os.path.exists(path):
        return None
    try:
        d = json.load(open(path))
        return d.get(kernel)
    except Exception:
        return None


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    return O


def cpu_model():
    """The host CPU's model name (lscpu, else /proc/cpuinfo)."""
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
        for line in out.splitlines():
            if line.startswith("Model name:"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def oracle_steps(O, xs, L, steps, first=0):
    """`steps` full FP64 oracle steps of the headline workload (both orders
    with forces, the WT grid, a deposit every 10 steps); returns seconds."""
    sw = O.make_sw("STEP", r0=3.9)
    g = O.Grid([[0, 1], [0, 1]], [200, 200], 0.01, 0.005, 9.0, 300.0, 8.617343e-5, True)
    t0 = time.perf_counter()
    for k in range(first, first + steps):
        x = xs[k % len(xs)]
        o4 = O.steinh_l(4, x, L, 3.9, sw)
        o6 = O.steinh_l(6, x, L, 3.9, sw)
        s = [o4["cv"], o6["cv"]]
        if k % 10 == 0:
            g.add_hill(s)
        V, dV = g.value(s)
        _ = -(dV[0] * o4["grad"] + dV[1] * o6["grad"])
    return time.perf_counter() - t0


def cpu_baseline(xs, L, budget_s=15.0, threads=None):
    """The FP64 oracle (C, OpenMP) running the same step on the host cores: as
    many full steps as fit the budget (at most 50) on `threads` threads, and
    one full step on one thread."""
    O = _oracle()
    n = xs[0].shape[0]
    if threads:
        O.set_threads(threads)
    cores = O.get_threads()
    oracle_steps(O, xs, L, 1)   # warm-up (page-in, thread pool)
    steps, el = 0, 0.0
    while el < budget_s and steps < 50:
        el += oracle_steps(O, xs, L, 1, first=steps)
        steps += 1
    O.set_threads(1)
    el1 = oracle_steps(O, xs, L, 1)
    O.set_threads(cores)
    return {"value": n * steps / el, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": "%d full steps of the 256,000-atom workload (FP64 oracle, both orders with forces, grid)" % steps,
            "cpu_model": cpu_model(), "cores_available": os.cpu_count(),
            "one_thread": {"value": n / el1, "unit": UNIT, "sample": "1 full step on 1 thread"}}


def error_vs_fp64(xs, L, precision, device):
    """Errors of one step of the timed workload against the FP64 oracle: a
    fresh context (deposit step 0) on the first positions; CVs and bias
    relative, forces relative to the largest force component, per-atom
    neighbour counts compared exactly.  Outside every timed region."""
    import mtd
    O = _oracle()
    x = xs[0]
    n = x.shape[0]
    m = mtd.Metad(fix_args(), precision=precision, device=device)
    m.set_box([0, 0, 0], L)
    f = np.zeros_like(x)
    m.post_force(0, x, f)
    st = O.make_sw("STEP", r0=3.9)
    o4, o6 = O.steinh_l(4, x, L, 3.9, st), O.steinh_l(6, x, L, 3.9, st)
    g = O.Grid([[0, 1], [0, 1]], [200, 200], 0.01, 0.005, 9.0, 300.0, 8.617343e-5, True)
    s = [o4["cv"], o6["cv"]]
    g.add_hill(s)
    V, dV = g.value(s)
    fo = -(dV[0] * o4["grad"] + dV[1] * o6["grad"])
    fmax = float(np.abs(fo).max())
    nnb = m.extract("Q4.nnb", n).astype(np.int32)
    out = {"precision": precision, "step": "0 (deposit)",
           "cv_rel": [abs(m.cv[d] - s[d]) / abs(s[d]) for d in range(2)],
           "bias_rel": abs(m.compute_scalar() - V) / abs(V),
           "force_rel_max": float(np.abs(f - fo).max()) / fmax,
           "force_rel_rms": float(np.sqrt(np.mean((f - fo) ** 2))) / fmax,
           "lq_rel_max": [float(np.abs(m.extract("Q%d.stein_q" % l, n) - o["LQ"]).max() / np.abs(o["LQ"]).max())
                          for l, o in ((4, o4), (6, o6))],
           "neighbor_counts_equal": bool(np.array_equal(nnb, o4["nnb"])),
           "cv_target_1e-6_met": bool(max(abs(m.cv[d] - s[d]) / abs(s[d]) for d in range(2)) <= 1e-6)}
    m.close()
    return out


def run_reference(args, rank):
    """The reference arm: the FP64 oracle port of the reference algorithm on
    all host cores, `warmup` untimed and exactly `steps` timed full steps of
    the headline workload; rank 0 alone (other ranks exit without work)."""
    if rank != 0:
        return 0
    xs, L = load_system()
    O = _oracle()
    cores = os.cpu_count() or 1
    O.set_threads(cores)
    n = xs[0].shape[0]
    oracle_steps(O, xs, L, args.warmup)
    el = oracle_steps(O, xs, L, args.steps, first=args.warmup)
    value = n * args.steps / el
    base = {"value": value, "unit": UNIT, "cores": O.get_threads(), "kind": "port",
            "sample": "%d full steps of the 256,000-atom workload after %d untimed (FP64 oracle, both orders "
                      "with forces, grid)" % (args.steps, args.warmup),
            "cpu_model": cpu_model()}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": el * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded slab geometry)",
            "config": {"workload": WORKLOAD, "atoms": int(n)},
            "cpu_baseline": base,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def secondary_workload(name):
    """The parity configs timed on request (`--workload sk|q`); the default
    workload above is the one the headline metric is quoted on."""
    import systems
    if name == "sk":
        x, L = systems.config3()
        args = ["GAUSSIAN", 0.05, 0.005, 10.0, "PACE", 10,
                "CAL", "NAME", "SK", "STRU_FACTOR_K", "all", "nk", 96, "kmag", systems.KMAG_111, "seed", 3,
                "SYMBOL", "v1", "SK.AVE", "CV_dim", 1, "DIM", 1, 0.0, 10.0, 2000, "v1", "WT", 0]
        desc = ("1,048,576-atom jittered FCC (a 5.26 A, sigma 0.2 A), k-vector S(k) over 96 directions on "
                "|k| = 2 pi sqrt(3)/a with forces, 1D 2000-bin grid, PACE 10")
        seeds = [(11, 0.2), (12, 0.2)]
    else:
        x, L = systems.config1()
        x = systems.jitter(x, 0.15, 2024)
        args = ["GAUSSIAN", 0.01, 0.005, 10.0, "PACE", 10,
                "CAL", "NAME", "Q6", "STEINH", "Q", 6, "all", "cutoff_r", 3.9, "cutoff_Natoms", 18,
                "SYMBOL", "v1", "Q6.AVE", "CV_dim", 1, "DIM", 1, 0.0, 1.0, 1000, "v1", "WT", 0]
        desc = "4,000-atom FCC (a 5.26 A, jitter 0.15 A), STEINH Q 6 cutoff 3.9 cap 18 with forces, 1D 1000-bin grid"
        seeds = [(21, 0.15), (22, 0.15)]
    base = systems.fcc(64, 5.26) if name == "sk" else systems.config1()[0]
    xs = [x] + [np.ascontiguousarray(systems.wrap(systems.jitter(base, sg, sd), L)) for sd, sg in seeds]
    xs = [np.ascontiguousarray(systems.wrap(v, L)) for v in xs]
    return args, xs, L, desc


def timing_stream():
    """A dedicated stream made torch's current one: the L2 flush, the
    library's kernels (set_stream) and the CUDA events all go to it, so each
    timed interval holds exactly one step, after the flush has completed."""
    import torch
    st = torch.cuda.Stream()
    torch.cuda.set_stream(st)
    return st


def kernel_profile(m, step_fn, flush, steps, stream):
    """Per-kernel durations from CUDA events recorded between the launches
    of `steps` steps.  The pass runs on its own stream: event intervals on the
    legacy default stream came out inflated by several microseconds per
    kernel, against per-kernel ncu durations of the same build."""
    import torch
    ps = torch.cuda.Stream()
    torch.cuda.synchronize()
    m.set_stream(ps.cuda_stream)
    m.profile(True)
    with torch.cuda.stream(ps):
        for _ in range(steps):
            flush.zero_()
            step_fn()
    m.sync()
    prof = m.profile_report()
    m.profile(False)
    m.set_stream(stream.cuda_stream)
    torch.cuda.synchronize()
    return prof


def run_secondary(args, local):
    import torch
    import mtd
    torch.cuda.set_device(local)
    fa, xs, L, desc = secondary_workload(args.workload)
    n = xs[0].shape[0]
    prec = "fp64" if args.workload == "q" else args.precision
    m = mtd.Metad(fa, precision=prec, device=local)
    m.set_box([0, 0, 0], L)
    m.init()
    stream = timing_stream()
    m.set_stream(stream.cuda_stream)
    dx = [torch.from_numpy(x).cuda() for x in xs]
    f = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    step = 0
    tuned = m.autotune(n, dx[0].data_ptr(), reps=3)   # shapes only: results do not depend on them
    for _ in range(args.warmup):
        m.post_force_device(step, n, dx[step % len(dx)].data_ptr(), f.data_ptr(), f.data_ptr())
        step += 1
    m.sync()

    def one_step():
        nonlocal step
        m.post_force_device(step, n, dx[step % len(dx)].data_ptr(), f.data_ptr(), f.data_ptr())
        step += 1

    prof = kernel_profile(m, one_step, flush, max(5, args.steps // 3), stream)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    hx = [torch.from_numpy(x).pin_memory() for x in xs]
    hf = torch.zeros((n, 3), dtype=torch.float64).pin_memory()
    with ClockSampler(local) as clk:
        t_end = time.perf_counter() + 0.6
        while time.perf_counter() < t_end:
            m.post_force_device(step, n, dx[step % len(dx)].data_ptr(), f.data_ptr(), f.data_ptr())
            step += 1
            m.sync()
        torch.cuda.synchronize()
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record(stream)
            m.post_force_device(step, n, dx[step % len(dx)].data_ptr(), f.data_ptr(), f.data_ptr())
            ev[k][1].record(stream)
            step += 1
        m.sync()
        torch.cuda.synchronize()
        dev_ms = sum(a.elapsed_time(b) for a, b in ev)
        m.set_stream(0)
        e2e_s = 0.0
        for k in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            hf.zero_()
            t0 = time.perf_counter()
            m.post_force(step, hx[step % len(hx)].numpy(), hf.numpy())
            e2e_s += time.perf_counter() - t0
            step += 1
    launches = m.launch_count()
    kernels = {k: v[1] / max(v[0], 1) for k, v in sorted(prof.items(), key=lambda kv: -kv[1][1])}
    line = {"metric": "CV+bias+force atom-steps/s", "workload": args.workload,
            "value": n * args.steps / (dev_ms / 1e3), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
            "dtype": "f32" if prec == "mixed" else "f64", "data": "synthetic (seeded)",
            "config": {"workload": desc, "atoms": n, "precision": prec,
                       "l2": "flushed (256 MB write) before each timed step", "cv": [float(v) for v in m.cv]},
            "e2e": {"value": n * args.steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 2 * 24 * n,
                    "d2h_bytes_per_step": 24 * n + 8 * 64, "ms_per_step": e2e_s * 1e3 / args.steps},
            "gpu_launches": launches * args.steps, "kernels_ms_per_step": kernels, "clocks": clk.summary(),
            "autotuned_shapes": {"neighbors_q_lambda": list(tuned), "sk_tiles": list(m.sk_tiles())}}
    if args.workload == "sk":
        pairs = n * 96
        ms = {k: v for k, v in kernels.items()}
        line["sk_pairs_per_s"] = {k: pairs / (v / 1e3) for k, v in ms.items() if k.startswith("sk_") and v > 0}
        line["roofline"] = sk_roofline(kernels, n, 96, clocks=line["clocks"])
    else:
        line["roofline"] = q_roofline(kernels, n)
    if not args.no_cpu:
        line["cpu_baseline"] = secondary_cpu_baseline(args.workload, xs, L)
    print(json.dumps(line))
    m.close()
    return 0


# Operations per (atom, k) pair of the S(k) passes, counted in the kernels'
# source (an FMA counts 2): FP64 -- the phase k.x (6) and its reduction to a
# quarter turn (5); FP32 -- the sin / cos polynomials (22), then the value
# pass accumulates cos and sin (2) and the force pass projects on rho(k) and
# k (9).
# per (atom, k): FP64 phase (k / pi).x (5) and half-turn reduction (3 adds);
# FP32 z^2, sin(pi z) (4 FMA + 1 mul), cos(pi z) (5 FMA), then the signed
# accumulation (2 FMA) or the force weight and gradient (1 mul + 1 FMA + 3 FMA)
SK_FLOP_PER_PAIR = {"sk_partial": {"fp64": 8, "fp32": 24}, "sk_force": {"fp64": 8, "fp32": 29}}


def sk_roofline(kernels, n, nk, clocks):
    """The S(k) passes are bound by arithmetic, not DRAM: achieved FP32 and
    FP64 rates of the dominant pass against the (non-tensor) peaks of the
    part at the sampled SM clock: 148 SMs x 128 FP32 lanes x 2 (FMA) x clock,
    and half that for FP64."""
    sk = {k: v for k, v in kernels.items() if k in SK_FLOP_PER_PAIR and v > 0}
    if not sk:
        return None
    name, ms = max(sk.items(), key=lambda kv: kv[1])
    mhz = (clocks or {}).get("sm_mhz") or 1965.0
    peak = 148 * 128 * 2 * mhz * 1e6 / 1e12
    per = SK_FLOP_PER_PAIR[name]
    a32 = per["fp32"] * n * nk / (ms / 1e3) / 1e12
    a64 = per["fp64"] * n * nk / (ms / 1e3) / 1e12
    peak_hbm, kind = peaks()
    bytes_ = n * 24 + 2 * 8 * nk * 1024   # positions once, per-block FP64 partials of rho(k)
    return {"bound": "fp32", "kernel": name, "achieved": a32, "peak": peak, "unit": "TFLOP/s",
            "frac": a32 / peak, "flop_per_pair": per, "avg_launch_ms": ms,
            "fp64": {"achieved": a64, "peak": peak / 2, "frac": a64 / (peak / 2)},
            "issue_frac": (a32 / peak) + (a64 / (peak / 2)),
            "peak_source": "148 SMs x 128 FP32 lanes x 2 x %.0f MHz (sampled); FP64 half of it" % mhz,
            "hbm": {"achieved": bytes_ / (ms / 1e3) / 1e9, "peak": peak_hbm, "unit": "GB/s",
                    "frac": bytes_ / (ms / 1e3) / 1e9 / peak_hbm, "peak_source": kind}}


def q_roofline(kernels, n):
    """Config 1 (4,000 atoms) is launch- and latency-bound: per-kernel
    durations of a few microseconds; the HBM fraction of the longest kernel
    is reported against the measured copy bandwidth."""
    if not kernels:
        return None
    name, ms = max(kernels.items(), key=lambda kv: kv[1])
    peak, kind = peaks()
    bytes_ = n * (24 + 4 * 18 + 2 * 7 * 8)   # positions, capped list, q_lm records (FP64, l = 6)
    return {"bound": "hbm", "kernel": name, "achieved": bytes_ / (ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
            "frac": bytes_ / (ms / 1e3) / 1e9 / peak, "peak_source": kind, "avg_launch_ms": ms,
            "note": "4,000 atoms: every kernel is a few microseconds; launch latency bounds the step"}


def secondary_cpu_baseline(workload, xs, L, budget_s=10.0):
    """The FP64 oracle (C, OpenMP) on the host cores for the same step: S(k)
    with forces (`sk`) or STEINH Q 6 with forces (`q`); grid work is negligible
    beside it and not timed."""
    import systems
    O = _oracle()
    O.set_threads(os.cpu_count())
    n = xs[0].shape[0]
    if workload == "sk":
        kv = systems.kvectors(96, systems.KMAG_111, 3)
        fn = lambda x: O.sk(x, kv, grad=True)
        desc = "S(k) over 96 k-vectors with forces, 1,048,576 atoms, FP64 oracle"
    else:
        fn = lambda x: O.steinh_q(6, x, L, 3.9, 18, grad=True)
        desc = "STEINH Q 6 (cutoff 3.9, cap 18) with forces, 4,000 atoms, FP64 oracle"
    fn(xs[0])
    steps, el = 0, 0.0
    while el < budget_s and steps < 200:
        t0 = time.perf_counter()
        fn(xs[steps % len(xs)])
        el += time.perf_counter() - t0
        steps += 1
    return {"value": n * steps / el, "unit": UNIT, "cores": O.get_threads(), "kind": "port",
            "sample": "%d full steps: %s" % (steps, desc), "cpu_model": cpu_model()}


def run_nnbias(args, local):
    """Learned 4D bias: 20,000 seeded hills (sigma 0.02, h 0.005 eV) along a 4D
    CV trajectory; the MLP is fitted on the device, checked on 65,536 sampled
    points, and the per-step bias (V and dV/ds at one CV point) is timed for
    the exact FP64 hill sum and for the network."""
    import torch
    import mtd
    import systems
    torch.cuda.set_device(local)
    c, h, sg = systems.cv4_hills(n=20000, seed=5)
    nb = mtd.NNBias(systems.CV4_LO, systems.CV4_HI, seed=3)
    nb.add_hills(c, h, sg)
    t0 = time.perf_counter()
    nb.fit(ntrain=262144, iters=args.nn_iters, batch=8192, lr=3e-3, seed=2)
    fit_s = time.perf_counter() - t0
    mx, rms = nb.validate(npts=65536, seed=7, tol=1e-3)
    stream = timing_stream()
    d_s = torch.tensor(c[len(c) // 2], dtype=torch.float64, device="cuda")
    d_v = torch.zeros(1, dtype=torch.float64, device="cuda")
    d_g = torch.zeros(4, dtype=torch.float64, device="cuda")
    res = {}
    for name, use in [("exact", 0), ("nn", 1)]:
        for _ in range(max(3, args.warmup)):
            nb.point_device(d_s.data_ptr(), d_v.data_ptr(), d_g.data_ptr(), use_nn=use, stream=stream.cuda_stream)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.steps):
            nb.point_device(d_s.data_ptr(), d_v.data_ptr(), d_g.data_ptr(), use_nn=use, stream=stream.cuda_stream)
        b.record(stream)
        torch.cuda.synchronize()
        res[name] = a.elapsed_time(b) * 1e3 / args.steps
    pts = systems.CV4_LO + (systems.CV4_HI - systems.CV4_LO) * np.random.default_rng(3).random((65536, 4))
    # V and dV/ds at 65,536 device-resident points: exact FP64 sum vs network,
    # CUDA events on the launching stream
    d_p = torch.from_numpy(np.ascontiguousarray(pts)).cuda()
    b_v = torch.zeros(len(pts), dtype=torch.float64, device="cuda")
    b_g = torch.zeros((len(pts), 4), dtype=torch.float64, device="cuda")
    batch = {}
    for name, use in [("exact", 0), ("nn", 1)]:
        reps = 3 if use == 0 else 20
        nb.eval_device(len(pts), d_p.data_ptr(), b_v.data_ptr(), b_g.data_ptr(), use_nn=use, stream=stream.cuda_stream)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            nb.eval_device(len(pts), d_p.data_ptr(), b_v.data_ptr(), b_g.data_ptr(), use_nn=use,
                           stream=stream.cuda_stream)
        b.record(stream)
        torch.cuda.synchronize()
        batch[name + "_us"] = a.elapsed_time(b) * 1e3 / reps
    batch["speedup"] = batch["exact_us"] / batch["nn_us"]
    # the same through the host-array calls (conversions, copies, allocations included)
    t0 = time.perf_counter()
    nb.exact(pts)
    ex_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    nb.eval(pts)
    nn_s = time.perf_counter() - t0
    # the exact sum grows with the hills deposited, the network does not
    scaling = {}
    for extra in [180000]:
        c2, h2, s2 = systems.cv4_hills(n=extra, seed=6)
        nb.add_hills(c2, h2, s2)
        for name, use in [("exact", 0), ("nn", 1)]:
            for _ in range(3):
                nb.point_device(d_s.data_ptr(), d_v.data_ptr(), d_g.data_ptr(), use_nn=use, stream=stream.cuda_stream)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for _ in range(args.steps):
                nb.point_device(d_s.data_ptr(), d_v.data_ptr(), d_g.data_ptr(), use_nn=use, stream=stream.cuda_stream)
            b.record(stream)
            torch.cuda.synchronize()
            scaling.setdefault(str(nb.num_hills), {})[name + "_us_per_step"] = a.elapsed_time(b) * 1e3 / args.steps
    line = {"metric": "learned 4D bias: bias V and dV/ds per MD step, exact FP64 hill sum vs MLP",
            "workload": "nn", "unit": "us/step", "higher_is_better": False,
            "exact_us_per_step": res["exact"], "nn_us_per_step": res["nn"],
            "speedup_per_step": res["exact"] / res["nn"], "per_step_vs_hills": scaling,
            "batch_65536_points_device": batch,
            "batch_65536_points_host_api_s": {"exact": ex_s, "nn": nn_s},
            "hills": int(len(h)), "vmax_eV": nb.vscale, "max_abs_err_eV": mx, "rms_err_eV": rms,
            "tolerance_eV": 1e-3, "tolerance_met": bool(mx <= 1e-3), "fit_s": fit_s,
            "fit": {"ntrain": 262144, "iters": args.nn_iters, "batch": 8192, "lr": 3e-3},
            "network": "4-128-128-1 SiLU, BF16 weights, FP32 accumulation (128x128 layer on tcgen05)",
            "params": 17281, "grid_equivalent_bytes": 8 * 200 ** 4, "steps": args.steps}
    print(json.dumps(line))
    nb.close()
    return 0


def tile_rank_positions(x0, L, world, rank, cut, seed, copies):
    """Rank `rank`'s atoms of the decomposed multi-GPU workload: `world`
    copies of the slab geometry tiled along x (tile t jittered with its own
    seed), rank r owning tile r and receiving as ghosts the atoms of the
    neighbouring tiles within `cut` of its faces (what LAMMPS's Comm
    supplies).  Returns the per-step position arrays (owned rows first, then
    ghosts, in tile-local coordinates), the number of owned atoms, and the
    box (lo, hi, periodic): x non-periodic and grown by `cut`, y and z
    periodic over the tile."""
    import systems
    Lx = L[0]

    def tile(t, c):
        # jittered, wrapped in y and z only: an atom of tile t stays tile t's
        # (ownership by tile, as between two reneighborings of an MD code)
        x = systems.jitter(x0, 0.05, seed + 1 + 1000 * (t % world), c)
        if world == 1:
            return systems.wrap(x, L)
        x[:, 1:] -= np.floor(x[:, 1:] / L[1:]) * L[1:]
        return x

    # the ghost atoms are chosen once (on the unjittered geometry, with a
    # margin above the jitter), as an MD code keeps its ghosts between
    # reneighborings; their positions follow every step
    margin = 0.5
    gi_r = np.nonzero(x0[:, 0] < cut + margin)[0]
    gi_l = np.nonzero(x0[:, 0] >= Lx - cut - margin)[0]
    out = []
    for c in range(copies):
        own = tile(rank, c)
        if world == 1:
            out.append(np.ascontiguousarray(own))
            continue
        gr = tile(rank + 1, c)[gi_r] + np.array([Lx, 0.0, 0.0])
        gl = tile(rank - 1, c)[gi_l] - np.array([Lx, 0.0, 0.0])
        out.append(np.ascontiguousarray(np.concatenate([own, gr, gl])))
    if world == 1:
        return out, out[0].shape[0], ([0.0, 0.0, 0.0], list(L), (1, 1, 1))
    return out, x0.shape[0], ([-cut, 0.0, 0.0], [Lx + cut, L[1], L[2]], (0, 1, 1))


def max_over_ranks(vals, dist, device):
    """Timings (ms) reduced to their maximum over the ranks (the slowest replica
    sets the job's time); identity without a process group."""
    import torch
    t = torch.tensor([float(v) for v in vals], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t]


def replica_throughput(n_atoms, steps, world, ms):
    """Whole-job atom-steps/s: every rank runs its own replica of n_atoms for
    `steps` steps (weak scaling, no data-path collective) within `ms`."""
    return n_atoms * steps * world / (ms / 1e3)


def walker_args():
    """The headline workload's CVs on a 256 x 256 WT grid (config of the
    multi-walker case); per-step neighbour lists (the persistent step kernel
    builds them inside its one launch)."""
    a = fix_args(skin=0)
    i = a.index("DIM")
    return a[:i] + ["DIM", 1, 0, 1, 256, "v1", "DIM", 2, 0, 1, 256, "v2", "WT", 1]


def run_walkers(args, local):
    """32 walkers, atom counts drawn from U{2000..64000} (seeded), FCC / disordered
    slabs, sharing one 2D WT grid; one MD step = every walker's CVs, the
    synchronous deposit and every walker's forces."""
    import torch
    import mtd
    import systems
    torch.cuda.set_device(local)
    rng = np.random.default_rng(44)
    ns = rng.integers(2000, 64001, size=32)
    syss = [systems.walker_system(int(n), 100 + k) for k, n in enumerate(ns)]
    ns = [x.shape[0] for x, _ in syss]
    res = {}
    modes = [("plain", False, False), ("graph", True, False), ("persistent", False, True),
             ("persistent_graph", True, True)]
    for mode, graph, persistent in modes:
        W = mtd.Walkers(len(syss), walker_args(), precision=args.precision)
        for k, (x, L) in enumerate(syss):
            W.set_box(k, [0, 0, 0], L)
        W.init()
        W.enable_graph(graph)
        W.enable_persistent(persistent)
        dx = [torch.from_numpy(np.ascontiguousarray(x)).cuda() for x, _ in syss]
        df = [torch.zeros_like(v) for v in dx]
        xp, fp = [v.data_ptr() for v in dx], [v.data_ptr() for v in df]
        picks = W.autotune(ns, xp, reps=5)   # kernel shapes per walker (results do not depend on them)
        step = 0
        for _ in range(max(3, args.warmup)):
            W.step_device(step, ns, xp, fp)
            W.sync()
            step += 1
        launches = W.launch_count()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            W.step_device(step, ns, xp, fp)
            W.sync()
            step += 1
        torch.cuda.synchronize()
        wall = (time.perf_counter() - t0) / args.steps
        shapes = {}
        for p in picks:
            key = "nbr%d/q%d/l%d" % p
            shapes[key] = shapes.get(key, 0) + 1
        res[mode] = {"ms_per_step": wall * 1e3, "atom_steps_per_s": sum(ns) / wall, "launches_per_step": launches,
                     "one_launch": bool(W.persistent_active)}
        if not persistent:
            res[mode]["autotuned_shapes"] = shapes
        cvs = [W.cv(k, 2).tolist() for k in range(3)]
        W.close()
    best = max(res, key=lambda k: res[k]["atom_steps_per_s"])
    line = {"metric": "multi-walker CV+bias+force atom-steps/s (all walkers)", "workload": "walkers",
            "value": res[best]["atom_steps_per_s"], "mode": best, "unit": UNIT, "higher_is_better": True,
            "steps": args.steps, "warmup": args.warmup, "walkers": len(ns), "atoms_total": int(sum(ns)),
            "atoms_min": int(min(ns)), "atoms_max": int(max(ns)), "precision": args.precision,
            "timing": "host wall clock per step including the per-step synchronisation and output collection",
            "modes": res, "cv_first_walkers": cvs,
            "config": "STEINH L Q4+Q6 STEP 3.9 A, MEAN_SOLID, shared 2D 256x256 WT grid, PACE 10"}
    print(json.dumps(line))
    return 0


def run_domain(args, local):
    """Per-step cost of the domain-decomposition exchange on the headline
    workload with one rank owning every atom (so the results equal the plain
    step): plain, host allreduce callback, device callback that enqueues
    nothing, device callback through a one-rank NCCL group.  Wall clock per
    synchronised step after an L2 flush (the exchange is host latency, which
    CUDA events on the device would not show)."""
    import socket
    import time

    import torch
    import torch.distributed as dist

    import domain
    import mtd
    torch.cuda.set_device(local)
    xs, L = load_system()
    n = xs[0].shape[0]
    dx = [torch.from_numpy(x).cuda() for x in xs]
    f = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % port, rank=0, world_size=1)
    res, cvs = {}, {}
    try:
        for mode in ("plain", "host", "device", "device_nccl"):
            m = mtd.Metad(fix_args(), precision=args.precision, device=local)
            if mode == "host":
                m.set_domain(n, 0, domain.LocalAllreduce(1).for_rank(0))
            elif mode == "device":
                m.set_domain_device(n, 0, lambda p, c, s: None)
            elif mode == "device_nccl":
                m.set_domain_device(n, 0, domain.TorchDeviceAllreduce())
            m.set_box([0, 0, 0], L)
            step = 0
            for _ in range(args.warmup):
                m.post_force_device(step, n, dx[step % len(dx)].data_ptr(), f.data_ptr(), f.data_ptr())
                step += 1
            m.sync()
            tot = 0.0
            for _ in range(args.steps):
                flush.zero_()
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                m.post_force_device(step, n, dx[step % len(dx)].data_ptr(), f.data_ptr(), f.data_ptr())
                m.sync()
                tot += time.perf_counter() - t0
                step += 1
            res[mode] = tot * 1e3 / args.steps
            cvs[mode] = m.cv.tolist()
            m.close()
    finally:
        dist.destroy_process_group()
    print(json.dumps({"metric": "domain-decomposition exchange cost", "workload": "domain", "unit": "ms/step",
                      "higher_is_better": False, "steps": args.steps, "warmup": args.warmup,
                      "ms_per_step": res, "exchange_us": {k: (v - res["plain"]) * 1e3 for k, v in res.items()},
                      "cv_equal": all(c == cvs["plain"] for c in cvs.values()),
                      "config": {"workload": WORKLOAD, "atoms": n, "ranks": 1,
                                 "timing": "wall clock per synchronised step after a 256 MB L2 flush"}}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--workload", default="local", choices=["local", "sk", "q", "nn", "walkers", "domain"],
                    help="local: the headline 256k-atom STEINH L workload; sk: 1M-atom k-vector S(k); "
                         "q: 4,000-atom STEINH Q (FP64); nn: learned 4D bias vs exact hill sum; "
                         "walkers: 32 walkers sharing one grid; domain: cost of the decomposition exchange")
    ap.add_argument("--nn-iters", type=int, default=20000, help="Adam steps of the learned-bias fit (--workload nn)")
    ap.add_argument("--split", default="domain", choices=["domain", "replicas"],
                    help="with several GPUs: domain decomposition of tiled slabs (per-step NCCL allreduce) or "
                         "independent replicas")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        return run_reference(args, rank)
    args.warmup = max(args.warmup, 3)
    if args.workload == "nn":
        return run_nnbias(args, local)
    if args.workload == "walkers":
        return run_walkers(args, local)
    if args.workload == "domain":
        return run_domain(args, local)
    if args.workload != "local":
        return run_secondary(args, local)

    import torch
    import mtd
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    xs, L = load_system()
    split = args.split if world > 1 else "none"
    nown = xs[0].shape[0]
    m = mtd.Metad(fix_args(), precision=args.precision, device=local)
    if split == "domain":
        # the reference's multi-rank model: tiles of the slab over the ranks,
        # ghosts from the neighbouring tiles, the per-step unit totals summed
        # over the ranks by NCCL on the library's stream
        import domain
        x0, _ = load_base(2024)
        cut = m.ghost_cutoff
        xs, nown, (blo, bhi, bper) = tile_rank_positions(x0, L, world, rank, cut, 2024, 4)
        m.set_domain_device(nown, rank, domain.TorchDeviceAllreduce())
        m.set_box(blo, bhi, bper)
    else:
        m.set_box([0, 0, 0], L)
    n = xs[0].shape[0]
    m.init()
    stream = timing_stream()
    m.set_stream(stream.cuda_stream)
    dx = [torch.from_numpy(x).cuda() for x in xs]
    f_in = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    f_out = torch.zeros_like(f_in)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    step = 0

    def dev_step():
        nonlocal step
        m.post_force_device(step, n, dx[step % len(dx)].data_ptr(), f_in.data_ptr(), f_out.data_ptr())
        step += 1

    for _ in range(args.warmup):
        dev_step()
    m.sync()
    # kernel shapes from the autotuner (every shape gives bitwise-identical steps)
    tuned = m.autotune(n, dx[0].data_ptr(), reps=5)
    for _ in range(2):
        dev_step()
    m.sync()
    torch.cuda.synchronize()
    launches = m.launch_count()
    nbar = None
    try:
        from scipy.spatial import cKDTree
        t = cKDTree(xs[0], boxsize=L)
        nbar = float((t.query_ball_point(xs[0], 3.9 - 1e-9, return_length=True) - 1).mean())
    except Exception:
        nbar = 8.0

    prof = kernel_profile(m, dev_step, flush, max(5, args.steps // 3), stream)

    hx = [torch.from_numpy(x).pin_memory() for x in xs]
    hf = torch.zeros((n, 3), dtype=torch.float64).pin_memory()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        # untimed pre-roll so the sampler is up and the clocks have ramped
        t_end = time.perf_counter() + 0.6
        while time.perf_counter() < t_end:
            dev_step()
            m.sync()
        # timed, device-resident
        if dist:
            dist.barrier()
        builds0 = m.neighbor_stats()[0]
        torch.cuda.synchronize()
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record(stream)
            dev_step()
            ev[k][1].record(stream)
        m.sync()
        torch.cuda.synchronize()
        dev_ms = sum(a.elapsed_time(b) for a, b in ev)
        builds_timed, skin_active = m.neighbor_stats()
        builds_timed -= builds0

        # e2e through the C ABI on pinned host buffers; the untimed calls
        # include the library's timing trial of the host copy modes (mode 0)
        m.set_stream(0)
        for k in range(12):
            hf.zero_()
            m.post_force(step, hx[step % len(hx)].numpy(), hf.numpy())
            step += 1
        copy_mode_used = m.host_copy_mode_in_use()
        e2e_s = 0.0
        for k in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            hf.zero_()
            t0 = time.perf_counter()
            m.post_force(step, hx[step % len(hx)].numpy(), hf.numpy())
            e2e_s += time.perf_counter() - t0
            step += 1
    clocks = clk.summary()
    # the three ways f can cross the host link (mtd_set_host_copy_mode), same forces
    copy_modes = {}
    for mode in (1, 2, 3):
        m.set_host_copy_mode(mode)
        t = 0.0
        for k in range(max(5, args.steps // 2)):
            flush.zero_()
            torch.cuda.synchronize()
            hf.zero_()
            t0 = time.perf_counter()
            m.post_force(step, hx[step % len(hx)].numpy(), hf.numpy())
            t += time.perf_counter() - t0
            step += 1
        copy_modes[{1: "copies", 2: "upload + zero-copy write", 3: "zero copy both ways"}[mode]] = \
            t * 1e3 / max(5, args.steps // 2)
    m.set_host_copy_mode(copy_mode_used or 0)
    # where the end-to-end step goes: the library's event marks around the
    # host copies and kernels of a few more calls (a separate, untimed pass)
    m.profile(True)
    for k in range(5):
        flush.zero_()
        torch.cuda.synchronize()
        hf.zero_()
        m.post_force(step, hx[step % len(hx)].numpy(), hf.numpy())
        step += 1
    e2e_split = {k: v[1] / max(v[0], 1) for k, v in sorted(m.profile_report().items(), key=lambda kv: -kv[1][1])}
    m.profile(False)

    dev_ms, e2e_ms = max_over_ranks([dev_ms, e2e_s * 1e3], dist, "cuda")
    # whole-job throughput counts owned atoms (ghosts are copies)
    value, e2e_value = replica_throughput(nown, args.steps, world, dev_ms), replica_throughput(nown, args.steps,
                                                                                              world, e2e_ms)

    # roofline of the dominant kernel
    peak, peak_kind = peaks()
    dom = max(prof.items(), key=lambda kv: kv[1][1])
    dom_name, (calls, tot_ms) = dom
    avg_ms = tot_ms / max(calls, 1)
    nbytes = kernel_bytes(dom_name, n, nbar)
    achieved = nbytes / (avg_ms / 1e3) / 1e9 if nbytes else None
    roof = {"bound": "hbm", "kernel": dom_name, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind,
            "traffic": ncu_traffic(dom_name), "avg_launch_ms": avg_ms,
            "algorithmic_bytes_per_launch": nbytes,
            "kernels_ms_per_step": {k: v[1] / max(v[0], 1) for k, v in sorted(prof.items(), key=lambda kv: -kv[1][1])},
            "pipeline": {"bytes_per_atom_step": pipeline_bytes(nbar),
                         "achieved": pipeline_bytes(nbar) * n / (dev_ms / args.steps / 1e3) / 1e9,
                         "frac": pipeline_bytes(nbar) * n / (dev_ms / args.steps / 1e3) / 1e9 / peak}}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(xs, L, budget_s=15.0, threads=os.cpu_count())
    err = None
    if rank == 0 and world == 1 and not args.no_cpu:
        err = error_vs_fp64(xs, L, args.precision, local)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if args.precision == "mixed" else "f64",
            "data": "synthetic (seeded FCC/BCC/liquid slabs, 4 jittered copies cycled)",
            "config": {"workload": WORKLOAD, "atoms": n, "mean_neighbors": nbar,
                       "max_neighbors": m.max_neighbors("Q4"), "cap_cutoff_Natoms": 18,
                       "precision": args.precision, "l2": "flushed (256 MB write) before each timed step",
                       "parallelism": {"none": "single GPU",
                                       "replicas": "%d independent replicas (no data-path collective)" % world,
                                       "domain": "domain decomposition over %d ranks: x tiles of the slab, ghost "
                                                 "shell %.1f A, per-step NCCL allreduce of the unit totals on the "
                                                 "library stream; ghost-force reverse communication is the MD "
                                                 "code's and is not timed" % (world, m.ghost_cutoff)}[split],
                       "atoms_per_rank": {"owned": int(nown), "with_ghosts": int(n)},
                       "autotuned_shapes": dict(m.tuning(), neighbors=["fast/256", "fast/128", "flat/128"][tuned[0]]),
                       "neighbor_lists": {"skin_A": SKIN, "rebuild_every_steps": EVERY,
                                          "rebuild_when_moved_A": SKIN / 2, "skin_active": skin_active,
                                          "rebuilds_in_timed_steps": builds_timed,
                                          "rule": "exact lists every step, filtered from candidates within "
                                                  "cutoff + skin; cell list and candidates rebuilt when an atom "
                                                  "moves more than skin/2 and at least every 10 steps"},
                       "cv": [float(v) for v in m.cv]},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 2 * 24 * n,
                    "d2h_bytes_per_step": 24 * n + 8 * 64, "ms_per_step": e2e_ms / args.steps,
                    "split_ms": e2e_split,
                    "copies": "x uploaded in 3 MB pieces; f (pinned) over the host link in the mode the "
                              "library's timing trial picked on the untimed calls (1: side-stream upload and a "
                              "download, 2: upload and zero-copy write, 3: zero copy both ways)",
                    "host_copy_mode": copy_mode_used,
                    "host_copy_modes_ms_per_step": copy_modes},
            "gpu_launches": launches * args.steps,
            "roofline": roof, "clocks": clocks, "cpu_baseline": cpu, "error_vs_fp64": err}
    if rank == 0:
        print(json.dumps(line))
    m.close()
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
