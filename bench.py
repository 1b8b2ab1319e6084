#!/usr/bin/env python
"""Benchmark of the B200 IBFS per-timestep advance (one JSON line on rank 0).

Workload (N=1): flat plate of chord 1 at 30 deg angle of attack, Re=300,
400x400 cells per level, 5 nested levels, dt=0.002, domain [-2,2]^2, body
points at spacing dx along the chord (101 points), stationary body with the
Cholesky force solve -- seeded synthetic input of that shape (the reference
runs no public dataset). A "step" is one full advance (operators.f90:62-188)
of that case. The unit is cell-updates/s: L*m*n cells advanced per step.

Timing: W untimed warm-up steps, then K steps, each preceded by an L2 flush
(a 256 MB device write; the case state is ~60 MB and would otherwise stay in
the 126 MB L2), each timed with CUDA events on the library's stream. `value`
is the device-timed throughput with the state resident in HBM; `e2e` is the
same metric through the public per-step call (ibfs_advance) with the body
velocities copied host->device from pinned memory and the forces / circulation
/ slip copied back every step, timed on the host clock.

`--impl reference` times the CPU restatement of the reference (the oracle,
a port: the Fortran+FFTW reference cannot be built here) on all host cores,
one independent case per process, on the same workload.

With torchrun (N>1) every rank runs an independent replica of the case
("replicas only": the path has no exchange step); value is the sum over ranks
of the cell-updates divided by the max over ranks of the device time.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ibfs-if2d_b200"))

METRIC = "cell-updates/s plain vs batched split-prec at ≤1e-8 force err; adjoint/fwd cost"
UNIT = "cell-updates/s"
WORKLOAD = dict(workload="flat plate 30deg, Re 300, 400x400 cells x 5 levels, dt 0.002, 101 body points",
                m=400, n=400, levels=5, re=300.0, dt=0.002, body="plate", aoa_deg=30.0, chord=1.0,
                domain="[-2,2]^2")


def plate_points(m, length=4.0, chord=1.0, aoa=30.0):
    """line() of the reference geometry primitives (grid.f90:431-462)."""
    pi = 3.1415926535897932384
    ds = length / m
    angle = -aoa * pi / 180.0
    npt = int(chord / ds)
    seg = np.arange(npt + 1, dtype=np.float64) * chord / float(npt)
    xb = -0.5 * chord * math.cos(angle) + seg * math.cos(angle)
    yb = -0.5 * chord * math.sin(angle) + seg * math.sin(angle)
    return xb, yb


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def count(self):
        try:
            return sum(1 for _ in open(self.path))
        except OSError:
            return 0

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9:
                    rows.append(f)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def run_ours(args):
    import torch
    import ibfs_capi as C

    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    W = WORKLOAD
    xb, yb = plate_points(W["m"])
    prec = 1 if args.form == "precision" else 0
    params = C.make_params(W["m"], W["n"], W["dt"], W["re"], W["levels"])
    g = C.Solver(params, (xb, yb), C.make_options(precision=prec))
    g.precompute()
    s = g.sizes[0]
    cells = s["nlev"] * W["m"] * W["n"]
    nf = s["nf"]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def one_step():
        flush.zero_()
        torch.cuda.synchronize()
        g.advance_n(1, want_hist=False)
        return g.last_ms()

    with ClockSampler(local) as cs:
        # warm-up steps; keep warming until the clock sampler has a sample, so
        # the record covers the timed region even when it is shorter than the
        # 200 ms sampling period
        t_end = time.time() + 5.0
        nw = 0
        while nw < args.warmup or (cs.count() < 1 and time.time() < t_end):
            one_step()
            nw += 1
        if pg:
            pg.barrier()
        torch.cuda.synchronize()
        times = [one_step() for _ in range(args.steps)]
        torch.cuda.synchronize()
        time.sleep(0.25)
    tot_ms = sum(times)
    if pg:
        t = torch.tensor([tot_ms], dtype=torch.float64, device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        tot_ms = float(t.item())
        pg.barrier()
    value = cells * args.steps * ws / (tot_ms / 1e3)
    ms_per_step = tot_ms / args.steps

    # per-class device time of one step (CUDA events around every launch)
    prof = g.profile_step()
    kern = g.kernels_per_step()

    out = None
    if rank == 0:
        # roofline of the dominant kernel class
        dom = max(prof, key=lambda k: prof[k]["ms"])
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except OSError:
            pass
        hbm = peaks.get("hbm_gbs", 6650.0)
        bf16 = peaks.get("bf16_tflops", 1590.0)
        peak_src = "of measured" if peaks else "of fallback"
        step_bytes = 64.0 * cells + 8.0 * nf * nf
        if dom in ("gemm_tc",):
            ach = prof[dom]["flops"] / (prof[dom]["ms"] / 1e3) / 1e12
            roof = {"bound": "tensor", "achieved": ach, "peak": bf16, "unit": "TFLOP/s", "frac": ach / bf16,
                    "traffic": None, "kernel": "tcgen05 split-BF16 sine-transform GEMM", "peak_source": peak_src}
        elif dom == "gemm_f64":
            # FP64 DFMA GEMM: no FP64 peak is measured on this pool; report its
            # algorithmic rate and the whole step against the HBM roofline.
            ach = step_bytes / (ms_per_step / 1e3) / 1e9
            roof = {"bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                    "traffic": None, "kernel": "whole step (64 B/cell-update + 8 Nf^2 B)",
                    "peak_source": peak_src,
                    "dominant_kernel": "k_gemm_f64 (FP64 DFMA sine-transform GEMM)",
                    "dominant_fp64_tflops": prof[dom]["flops"] / (prof[dom]["ms"] / 1e3) / 1e12,
                    "dominant_share": prof[dom]["ms"] / sum(v["ms"] for v in prof.values())}
        else:
            ach = step_bytes / (ms_per_step / 1e3) / 1e9
            roof = {"bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                    "traffic": None, "kernel": dom, "peak_source": peak_src}
        tr = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tr):
            try:
                roof["traffic"] = json.load(open(tr)).get(roof.get("kernel_key", dom))
            except (OSError, ValueError):
                pass

        e2e = None
        cpu = None
        if ws == 1:
            # end to end through the public per-step call, host buffers
            import ctypes
            vel = np.zeros(nf)
            hv = torch.zeros(nf, dtype=torch.float64).pin_memory()
            e2e_s = 0.0
            for _ in range(args.steps):
                flush.zero_()
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                vel[:] = hv.numpy()
                o = g.advance(body_vel=vel)
                e2e_s += time.perf_counter() - t0
            d2h = 8 * (2 * s["nbody"] + s["nlev"] + 1)
            e2e = {"value": cells * args.steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 8 * nf,
                   "d2h_bytes_per_step": d2h}
            # CPU baseline: the oracle on one host core, from the GPU's state
            cpu = cpu_baseline_sample(g, params, xb, yb, cells, args.cpu_steps)

        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if prec == 0 else "bf16x3+f64",
            "data": "synthetic (seeded geometry of the named config; no dataset)",
            "config": dict(WORKLOAD, form="plain FP64" if prec == 0 else "split-precision",
                           l2="flushed between timed steps (256 MB write)",
                           parallelism="replicas" if ws > 1 else "single GPU"),
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": kern * args.steps,
            "kernels_per_step": kern, "profile_step": prof, "clocks": cs.summary(),
            "impl": "ours",
        }
        print(json.dumps(out), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return out


def cpu_baseline_sample(g, params, xb, yb, cells, steps):
    """Time the oracle (CPU restatement, one core) on a bounded sample of the
    same workload, started from the GPU's current state and Cholesky factor."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    p = O.make_params(params.m, params.n, params.dt, params.re, params.mgridlev, istart=1)
    c = O.Case(p, xb, yb)
    cm, cv = g.get_cholesky()
    c.set_cholesky(cm, cv)
    st = g.get_state()
    c.set_state(**{k: np.ascontiguousarray(v) for k, v in st.items()})
    t0 = time.perf_counter()
    for _ in range(steps):
        c.advance()
    dt = time.perf_counter() - t0
    return {"value": cells * steps / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{steps} steps of the same case on 1 host core (oracle/ibfs_oracle.c, own FFT DST-I), "
                      f"from the GPU's state; {dt:.1f} s"}


def _ref_worker(args):
    steps, warmup, seed = args
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    W = WORKLOAD
    xb, yb = plate_points(W["m"])
    c = O.Case(O.make_params(W["m"], W["n"], W["dt"], W["re"], W["levels"]), xb, yb)
    for _ in range(warmup):
        c.advance()  # first step runs preprocess (untimed), as advance does at itime==1
    t0 = time.perf_counter()
    for _ in range(steps):
        c.advance()
    return time.perf_counter() - t0, W["levels"] * W["m"] * W["n"] * steps


def run_reference(args):
    ws, rank, local = dist_setup()
    if rank != 0:
        return None
    import multiprocessing as mp
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.build()
    ncores = os.cpu_count() or 1
    procs = max(1, min(ncores, args.ref_procs))
    steps = max(1, min(args.steps, args.ref_steps))
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        res = pool.map(_ref_worker, [(steps, max(1, args.warmup), i) for i in range(procs)])
    tmax = max(r[0] for r in res)
    cells = sum(r[1] for r in res)
    value = cells / tmax
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": steps, "warmup": args.warmup,
        "ms_per_step": tmax / steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded geometry of the named config; no dataset)",
        "config": dict(WORKLOAD, form="CPU restatement (oracle port)", parallelism=f"{procs} processes"),
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": "port",
                         "sample": f"{procs} independent cases x {steps} steps after {max(1, args.warmup)} "
                                   f"warm-up steps (first one runs the Cholesky preprocess)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="plain", choices=["plain", "precision"])
    ap.add_argument("--cpu-steps", type=int, default=12)
    ap.add_argument("--ref-procs", type=int, default=128)
    ap.add_argument("--ref-steps", type=int, default=20)
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
