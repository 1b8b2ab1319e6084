#!/usr/bin/env python
"""Benchmark of the B200 IBFS per-timestep advance (one JSON line on rank 0).

Metric: cell-updates/s (one cell of one level advanced one timestep; L*m*n per
case-step) of the plain FP64 GPU advance and of the batched split-precision
advance at <= 1e-8 relative force error, plus the cost of the discrete adjoint
relative to a forward solve.

Default workload (--form batch, the headline `value`): 256 independent
stationary cases advanced together, grids drawn from {128,192,256,384,512}^2
with 2-5 nested levels, Re log-uniform in [50,500], cylinder (D=1) or flat
plate (chord 1, angle of attack in [0,40] deg) with body-point spacing ~dx,
dt at CFL 0.4, FP64 Cholesky force solve per case, seed 20261203 -- seeded
synthetic cases of those shapes (the reference runs no public dataset). A
"step" is one advance (operators.f90:62-188) of all 256 cases: one replay of
the captured step graph, every sine transform a split-BF16 tcgen05 GEMM plus
one FP64 refinement sweep.

Timing: W untimed warm-up steps, then K steps timed with CUDA events on the
library's stream (ibfs_last_timing). The resident state is ~9 GB, far above
the 126 MB L2, so no flush is needed between steps. `e2e` is the same metric
through the public per-step call ibfs_batch_advance with host buffers: every
step copies all cases' body velocities host->device and the step's outputs
(forces, circulation, slip) device->host, timed on the host clock.

Beside the headline (N=1 only): the plain FP64 advance on the 400x400x5 flat
plate at 30 deg (Re 300, dt 0.002; L2 flushed between steps) and its ratio to
the headline, the batched FP64 advance of the same 256 cases, the split-vs-FP64
force and field errors, a sequential sample (cases one handle at a time), the
split-precision plate, the adjoint/forward cost on the rotating cylinder
(Re 150, 256x256x4, 126 points), 32 pitching plates advanced together
(512x512x5, CG force solve every step), and the adjoint/forward cost of the
mean-drag derivative w.r.t. the pitch amplitude on one such plate and on all
32 differentiated together.

`--impl reference` times the CPU restatement of the reference (the oracle, a
port: the Fortran+FFTW reference cannot be built here) on all host cores, one
independent case per process, on a bounded sample of the same batch.

With torchrun (N>1) every rank advances its own copy of the batch ("replicas
only": the path has no exchange step); value is the sum over ranks of the
cell-updates divided by the max over ranks of the device time.
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

import workloads as W  # noqa: E402

METRIC = "cell-updates/s plain vs batched split-prec at ≤1e-8 force err; adjoint/fwd cost"
UNIT = "cell-updates/s"
SEED = 20261203
BATCH = dict(workload="256 independent stationary cases, m in {128,192,256,384,512}, 2-5 levels, "
                      "Re log-uniform [50,500], cylinder or plate (AoA U[0,40] deg), ds~dx, dt at CFL 0.4",
             ncases=256, seed=SEED)
PLATE = dict(workload="flat plate 30 deg, Re 300, 400x400 cells x 5 levels, dt 0.002, 101 body points",
             m=400, levels=5, re=300.0, dt=0.002)


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


def max_over_ranks(x, pg):
    """Device time of the slowest rank (every rank calls this, in the same
    order, so the collective sequence stays identical across ranks)."""
    if pg is None:
        return float(x)
    import torch
    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def aggregate(cells_per_rank_step, steps, ws, tot_ms):
    """Whole-job throughput: the cell-updates of all ranks over the slowest
    rank's device time."""
    return cells_per_rank_step * steps * ws / (tot_ms / 1e3)


def peaks():
    try:
        p = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return p, "of measured"
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "of fallback"


def force_hist(g, hist, ncase):
    fx = np.array([[g.outputs_of(hist[s], i)["fx"][0] for s in range(hist.shape[0])] for i in range(ncase)])
    fy = np.array([[g.outputs_of(hist[s], i)["fy"][0] for s in range(hist.shape[0])] for i in range(ncase)])
    return fx, fy


def force_err(fx1, fy1, fx0, fy0):
    """Relative lift/drag error per case, in two norms:
    history: max over the steps of max(|dCd|, |dCl|) / max over the steps of
    |(Cd, Cl)| -- the error of the force history relative to its size;
    per step: max over the steps of max(|dCd|, |dCl|) / |(Cd, Cl)| of the same
    step -- stricter, since the impulsive start makes the first step's force
    hundreds of times the settled one. Returns the max and median over cases of
    each: (hist_max, hist_median, step_max, step_median)."""
    d = np.maximum(np.abs(fx1 - fx0), np.abs(fy1 - fy0))
    mag = np.sqrt(fx0 ** 2 + fy0 ** 2)
    hist = d.max(axis=1) / mag.max(axis=1)
    step = (d / mag).max(axis=1)
    return float(hist.max()), float(np.median(hist)), float(step.max()), float(np.median(step))


def algorithmic_transform_flops(cases, nlev):
    """Algorithmic sine-transform work of one step of the batch: the
    reference's 7L+2 two-dimensional DSTs per case-step (operators.f90:62-188;
    3 per level in the Crank-Nicolson update, 2 per level in each of the two
    vort2flux calls, 2 in ainv), each 2 (m-1)(n-1)[(m-1)+(n-1)] flops as a
    pair of dense sine-matrix products, unpadded."""
    tot = 0.0
    for c, L in zip(cases, nlev):
        M, N = c["m"] - 1, c["n"] - 1
        tot += (7 * L + 2) * 2.0 * M * N * (M + N)
    return tot


def issued_tensor_flops(cases, nlev):
    """Slice products actually issued per step by the split form (default
    refinement): every solve is 4 GEMMs of 6 products (first pass) plus 4 of
    the correction's products -- 6 for the 2L Poisson solves of the two
    vort2flux calls, 3 for the L Crank-Nicolson solves and ainv -- on
    128-row and 128-column padded tiles with K padded to 64 (the single-CTA
    tiles; a launch group on the 256 x 256 CTA-pair tile pads some grids
    further, so this is a lower bound there)."""
    rup = lambda x, a: (x + a - 1) // a * a
    tot = 0.0
    for c, L in zip(cases, nlev):
        N = c["m"] - 1
        per_product = 4 * 2.0 * rup(N, 128) ** 2 * rup(N, 64)
        tot += per_product * (2 * L * (6 + 6) + (L + 1) * (6 + 3))
    return tot


def roofline_gemm(prof, alg_flops, issued_flops, pk, src):
    """tcgen05 GEMM class: the step's algorithmic DST flops (the reference's
    7L+2 transforms per case-step) over the device time of the step's GEMM
    launches, i.e. algorithmic flops per launch / average launch time, against
    the sustained dense BF16 peak (the kernel runs inside a long step). The
    split form's slice products and refinement transforms are reported as
    `issued`, not as algorithmic work."""
    d = prof["gemm_tc"]
    if d["launches"] == 0 or d["ms"] <= 0:
        return None
    secs = d["ms"] / 1e3
    ach = alg_flops / secs / 1e12
    peak = pk.get("bf16_tflops_sustained", pk.get("bf16_tflops"))
    roof = {"bound": "tensor", "achieved": ach, "peak": peak, "unit": "TFLOP/s", "frac": ach / peak,
            "traffic": None, "kernel": "k_gemm_tc_persist + k_gemm_tc_pair (split-BF16 tcgen05 sine-transform GEMM; "
                      "single-CTA or CTA-pair tile per launch group, by the autotuner)",
            "peak_source": f"{src} (bf16 sustained)",
            "basis": "algorithmic = (7L+2) DSTs per case-step x 2(m-1)(n-1)[(m-1)+(n-1)] flops, unpadded",
            "launches_per_step": d["launches"], "avg_launch_us": d["ms"] / d["launches"] * 1e3,
            "algorithmic_flops_per_launch": alg_flops / d["launches"],
            "issued_tflops": issued_flops / secs / 1e12, "issued_frac": issued_flops / secs / 1e12 / peak,
            "issued_flops_per_step": issued_flops,
            "share_of_step": d["ms"] / sum(v["ms"] for v in prof.values())}
    tr = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tr):
        try:
            t = json.load(open(tr)).get("k_gemm_tc_persist_batch256")
            if t:
                roof["traffic"] = t["bytes_per_launch"]
                roof["traffic_note"] = t.get("note")
        except (OSError, ValueError):
            pass
    return roof


def cpu_sample_from_gpu(g, cases, ids, steps):
    """The oracle (CPU restatement, one host core) on a bounded sample of the
    batch: the given cases, started from the GPU's state and Cholesky factor."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    cells, secs = 0, 0.0
    for i in ids:
        c = cases[i]
        L = g.sizes[i]["nlev"]
        oc = O.Case(O.make_params(c["m"], c["n"], c["dt"], c["re"], c["levels"], istart=1), c["xb"], c["yb"])
        cm, cv = g.get_cholesky(i)
        oc.set_cholesky(cm, cv)
        st = g.get_state(i)
        oc.set_state(**{k: np.ascontiguousarray(v) for k, v in st.items()})
        t0 = time.perf_counter()
        for _ in range(steps):
            oc.advance()
        secs += time.perf_counter() - t0
        cells += L * c["m"] * c["n"] * steps
    return {"value": cells / secs, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{len(ids)} cases of the batch (ids {ids}) x {steps} steps each on 1 host core "
                      f"(oracle/ibfs_oracle.c, own FFT DST-I), from the GPU's state and factor; {secs:.1f} s"}


def plain_and_split_plate(C, torch, steps, warmup, flush):
    """Plain FP64 advance of the 400x400x5 plate (the comparison point of the
    metric), and the split-precision form of the same case with its Cd/Cl and
    per-level vorticity errors against FP64 over a fixed horizon."""
    c = W.plate_re300()
    params, bodies, _ = W.solver_args([c], C, 0)
    out = {}
    hs = {}
    for prec in (0, 1):
        g = C.Solver(params[0], bodies[0], C.make_options(precision=prec))
        g.precompute()
        nlev_plate = g.sizes[0]["nlev"]
        cells = nlev_plate * c["m"] * c["n"]
        horizon = 40
        hs[prec] = (g.advance_n(horizon), g.get_state())
        times = []
        for s in range(warmup + steps):
            flush.zero_()
            torch.cuda.synchronize()
            if s >= warmup:  # lets a profiler select the timed steps of each form
                torch.cuda.nvtx.range_push(f"plate_timed_{'fp64' if prec == 0 else 'split'}")
            g.advance_n(1, want_hist=False)
            if s >= warmup:
                torch.cuda.synchronize()
                torch.cuda.nvtx.range_pop()
                times.append(g.last_ms())
        ms = sum(times) / len(times)
        out[prec] = {"value": cells / (ms / 1e3), "ms_per_step": ms, "cells_per_step": cells,
                     "kernels_per_step": g.kernels_per_step(), "profile_step": g.profile_step()}
        g.close()
    (h0, s0), (h1, s1) = hs[0], hs[1]
    fx0, fy0 = h0[:, 0], h0[:, 1]
    fx1, fy1 = h1[:, 0], h1[:, 1]
    cd = np.abs(fx0).max()
    L = nlev_plate
    om0, om1 = s0["omega"].reshape(L, -1), s1["omega"].reshape(L, -1)  # omega(2:m,2:n,L), level slowest
    q0_, q1_ = s0["q"].reshape(L, -1), s1["q"].reshape(L, -1)

    def rel_max(a, b):
        return float(np.abs(a - b).max() / np.abs(b).max())

    def rel_l2(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    per_level = [rel_max(om1[k], om0[k]) for k in range(L)]
    field_err = {"omega_rel_l2_per_level": [rel_l2(om1[k], om0[k]) for k in range(L)],
                 "q_rel_max_per_level": [rel_max(q1_[k], q0_[k]) for k in range(L)],
                 "q_rel_l2_per_level": [rel_l2(q1_[k], q0_[k]) for k in range(L)]}
    plain = dict(out[0], workload=PLATE["workload"], form="plain FP64",
                 l2="flushed between timed steps (256 MB write)")
    split = dict(out[1], workload=PLATE["workload"], form="split-precision (single case)",
                 err_vs_fp64={"steps": 40, "cd_rel_max": float(np.abs(fx1 - fx0).max() / cd),
                              "cl_rel_to_max_cd": float(np.abs(fy1 - fy0).max() / cd),
                              "omega_rel_max_per_level": per_level, **field_err})
    return plain, split


def _force_errors(h1, h0, rows, history=False):
    """Relative force error of history h1 against h0 (columns rows = (fx, fy)):
    per step, max(|dCd|, |dCl|) / |(Cd, Cl)| of that step; with history=True
    divided by the largest |(Cd, Cl)| of the whole history instead."""
    fx1, fy1 = h1[:, rows[0]], h1[:, rows[1]]
    fx0, fy0 = h0[:, rows[0]], h0[:, rows[1]]
    mag = np.sqrt(fx0 ** 2 + fy0 ** 2)
    return np.maximum(np.abs(fx1 - fx0), np.abs(fy1 - fy0)) / (mag.max() if history else mag)


def _level_errors(s1, s0, L):
    out = {}
    for k in ("omega", "q"):
        a, b = s1[k].reshape(L, -1), s0[k].reshape(L, -1)
        out[k + "_rel_max_per_level"] = [float(np.abs(a[l] - b[l]).max() / np.abs(b[l]).max()) for l in range(L)]
        out[k + "_rel_l2_per_level"] = [float(np.linalg.norm(a[l] - b[l]) / np.linalg.norm(b[l])) for l in range(L)]
    return out


def split_error_long_horizon(C, plate_steps=5000, batch_steps=1000):
    """The split-precision form beside the plain FP64 form over the configured
    horizons: the 400x400x5 plate for its 5000 steps, and one case of every
    (m, L) stratum of the 256-case batch (plates and cylinders alternately)
    for its 1000 steps, advanced together. Force errors per step against the
    FP64 run (max(|dCd|, |dCl|) / |(Cd, Cl)|), their maximum and the step where
    it occurs; per-level omega and q errors at the end (max-abs relative and
    relative L2). Both forms start from rest with their own Cholesky factor."""
    out = {}
    c = W.plate_re300()
    params, bodies, _ = W.solver_args([c], C, 0)
    hist, state = {}, {}
    for prec in (0, 1):
        g = C.Solver(params[0], bodies[0], C.make_options(precision=prec))
        hist[prec] = g.advance_n(plate_steps)
        state[prec] = g.get_state()
        L = g.sizes[0]["nlev"]
        g.close()
    # the flow's own sensitivity: the plain FP64 advance again with another
    # summation order of its transforms (unsplit 32x32 tiles against the
    # split-K tiles the tuner gives a single case), a perturbation of ~1e-16
    g = C.Solver(params[0], bodies[0], C.make_options(precision=0, tile_cfg=1))
    h_alt = g.advance_n(plate_steps)
    g.close()
    fr = _force_errors(h_alt, hist[0], (0, 1))
    fe = _force_errors(hist[1], hist[0], (0, 1))
    marks = [s for s in (1, 10, 100, 1000, 2000, 3000, 4000, 5000) if s <= plate_steps]
    out["plate400_fp64_summation_order"] = {
        "steps": plate_steps, "force_err_max": float(fr.max()),
        "force_err_at": {str(s): float(fr[s - 1]) for s in marks},
        "basis": "plain FP64 with unsplit 32x32 transform tiles vs plain FP64 with the split-K tiles: the "
                 "growth of a round-off perturbation over the horizon"}
    out["plate400"] = {"workload": PLATE["workload"], "steps": plate_steps, "force_err_max": float(fe.max()),
                       "force_err_history_norm_max": float(_force_errors(hist[1], hist[0], (0, 1), True).max()),
                       "force_err_argmax_step": int(fe.argmax()) + 1,
                       "force_err_at": {str(s): float(fe[s - 1]) for s in marks},
                       **_level_errors(state[1], state[0], L)}
    cases = W.batch(BATCH["ncases"], seed=SEED)
    ids, _ = W.stratified_sample(cases)
    for label, cfl_scale in (("batch_sample", 1.0), ("batch_sample_cfl0.2", 0.5)):
        sample = [dict(cases[i], dt=cases[i]["dt"] * cfl_scale) for i in ids]
        hist, states, g0 = {}, {}, None
        for prec in (0, 1):
            p, b, o = W.solver_args(sample, C, prec)
            g = C.Solver(p, b, o)
            hist[prec] = g.advance_n(batch_steps)
            states[prec] = [g.get_state(i) for i in range(len(sample))]
            if prec == 0:
                g0 = g
                continue
            per = []
            for i in range(len(sample)):
                nb = len(g0.outputs_of(hist[0][0], i)["fx"])
                off = C.lib().ibfs_output_offset(g.h, i)
                f0 = hist[0][:, off:off + 2 * nb]
                row = {"id": ids[i], "m": sample[i]["m"], "levels": g.sizes[i]["nlev"], "body": sample[i]["body"]}
                if not np.isfinite(f0).all() or np.abs(f0).max() > 1e6:
                    bad = np.where(~np.isfinite(f0).all(axis=1) | (np.abs(f0).max(axis=1) > 1e6))[0]
                    row["fp64_diverged_at_step"] = int(bad[0]) + 1
                else:
                    fe = _force_errors(hist[1], hist[0], (off, off + nb))
                    row["force_err_history_norm"] = float(_force_errors(hist[1], hist[0], (off, off + nb), True).max())
                    lv = _level_errors(states[1][i], states[0][i], g.sizes[i]["nlev"])
                    row.update({"force_err_max": float(fe.max()), "force_err_argmax_step": int(fe.argmax()) + 1,
                                "omega_rel_max": max(lv["omega_rel_max_per_level"]),
                                "q_rel_max": max(lv["q_rel_max_per_level"])})
                per.append(row)
            ok = [x for x in per if "force_err_max" in x]
            out[label] = {"steps": batch_steps, "dt": f"{cfl_scale} x the workload's dt (CFL {0.4 * cfl_scale:.1f})",
                          "cases": per, "finite_cases": len(ok), "diverged_cases": len(per) - len(ok),
                          "force_err_max": max((x["force_err_max"] for x in ok), default=None),
                          "force_err_history_norm_max": max((x["force_err_history_norm"] for x in ok), default=None),
                          "omega_rel_max": max((x["omega_rel_max"] for x in ok), default=None),
                          "q_rel_max": max((x["q_rel_max"] for x in ok), default=None),
                          "sample": "one case per (m, L) stratum of the 256-case batch, plates and cylinders "
                                    "alternately; a case whose FP64 run diverges (as the oracle does at the "
                                    "workload's CFL 0.4 for some cases) is listed with the step, not compared"}
            g.close()
            g0.close()
    out["basis"] = ("split-precision GPU advance vs plain FP64 GPU advance (itself within 1e-10 of the oracle), "
                    "same inputs, per-step force error max(|dCd|,|dCl|)/|(Cd,Cl)|")
    return out


MAX_PITCH_STEP = 1000  # t = 1/(4 f) = 1 s at dt 0.001, f 0.25: alpha(t) = amplitude


def pitching_args(C, cases):
    """Solver arguments of pitching cases that start from rest at the phase of
    maximum pitch (istart = 1000), where the plates sit at their full
    amplitude and the CG force solve needs the most iterations."""
    params, bodies, opts = W.solver_args(cases, C)
    for p in params:
        p.istart = MAX_PITCH_STEP
    return params, bodies, opts


def pitch_cg_at_max_amplitude(C, steps=4, amp=30.0):
    """One config-5 plate at the batch's largest amplitude (30 deg), advanced
    from rest at the phase of maximum pitch: CG iterations and ms per step of
    the reference's unpreconditioned CG (cjgr) and of the CG preconditioned by
    factors of the force operator at a grid of pitch angles, turned with the
    plate."""
    out = {}
    for pre in (0, 1):
        params, bodies, opts = pitching_args(C, [W.pitching(amp_deg=amp, precond=bool(pre))])
        g = C.Solver(params[0], bodies[0], opts[0])
        its, ms = [], []
        for _ in range(steps):
            g.advance_n(1, want_hist=False)
            its.append(g.last_cg_iterations())
            ms.append(g.last_ms())
        g.close()
        out["precond" if pre else "reference_cg"] = {"cg_iterations": its, "ms_per_step": ms}
    out["workload"] = (f"plate pitching {amp} deg about mid-chord, Re 500, 512x512 cells x 5 levels, dt 0.001, "
                       "FP64 CG to relative 1e-12, from rest at t = 1 s (alpha = amplitude)")
    return out


def pitching_batch(C, steps=3, warmup=2):
    """Config-5 shape: 32 flat plates pitching about mid-chord with amplitudes
    U[5, 30] deg, Re 500, 512x512 cells x 5 levels, dt 0.001, FP64 CG force
    solve to a relative residual of 1e-12 every step, advanced together."""
    cases = W.pitching_batch(32, seed=SEED)
    params, bodies, opts = pitching_args(C, cases)
    g = C.Solver(params, bodies, opts)
    g.advance_n(warmup, want_hist=False)
    g.advance_n(steps, want_hist=False)
    ms = g.last_ms() / steps
    cells = W.cells_per_step(cases, [s["nlev"] for s in g.sizes])
    out = {"value": cells / (ms / 1e3), "unit": UNIT, "ms_per_step": ms, "steps": steps,
           "cg_iterations_last_step": g.last_cg_iterations(), "kernels_per_step_outside_cg": g.kernels_per_step(),
           "workload": "32 pitching plates (amplitude U[5,30] deg, f 0.25, mid-chord pivot), Re 500, "
                       "512x512 cells x 5 levels, dt 0.001, FP64 CG to relative residual 1e-12 preconditioned by "
                       "factors at a grid of pitch angles, from rest at t = 1 s (maximum pitch)"}
    g.close()
    return out


def pitch_adjoint_cost(C, steps=12, K=6, amp=20.0):
    """Config-5 grid (plate pitching about mid-chord, Re 500, 512x512 cells x 5
    levels, dt 0.001, FP64 CG to a relative 1e-12): the discrete adjoint of the
    mean drag over the last half of the horizon w.r.t. the pitch amplitude;
    cost = device time of the gradient run / device time of a plain forward
    run of the same steps from the same state."""
    case = W.pitching(amp_deg=amp)
    p, b, o = pitching_args(C, [case])
    f = C.Solver(p[0], b[0], o[0])
    f.advance_n(steps, want_hist=False)
    ms_plain = f.last_ms()
    f.close()
    g = C.Solver(p[0], b[0], o[0])
    wx = np.zeros(steps)
    wx[steps - steps // 2:] = 1.0 / (steps // 2)
    J, dJ, mf, mt = g.adjoint_pitch_run(steps, K, wx, np.zeros(steps))
    it = g.last_cg_iterations()
    g.close()
    return {"cost_ratio": mt / ms_plain, "cost_ratio_vs_own_forward_pass": mt / mf, "ms_total": mt,
            "ms_forward_pass": mf, "ms_plain_forward": ms_plain, "steps": steps, "checkpoint_every": K,
            "J": J, "dJ_damp_per_deg": dJ, "adjoint_cg_iterations_max": it,
            "workload": f"plate pitching {amp} deg about mid-chord, f 0.25, Re 500, 512x512 cells x 5 levels, "
                        f"dt 0.001, preconditioned FP64 CG to relative 1e-12, from rest at t = 1 s; J = mean drag "
                        f"over the last {steps // 2} steps, derivative w.r.t. the pitch amplitude"}


def pitch_adjoint_batch(C, steps=4, K=2):
    """Config 5 as specified: 32 plates pitching about mid-chord, amplitudes
    U[5, 30] deg, 512x512 cells x 5 levels, dt 0.001, FP64 CG to relative
    1e-12, advanced together, with the adjoint of each plate's mean drag (last
    half of the horizon) w.r.t. its amplitude, all 32 differentiated together;
    cost = device time of the gradient run / device time of a plain batched
    forward run of the same steps."""
    cases = W.pitching_batch(32, seed=SEED)
    params, bodies, opts = pitching_args(C, cases)
    f = C.Solver(params, bodies, opts)
    f.advance_n(steps, want_hist=False)
    ms_plain = f.last_ms()
    f.close()
    g = C.Solver(params, bodies, opts)
    wx = np.zeros(steps)
    wx[steps - steps // 2:] = 1.0 / (steps // 2)
    J, dJ, mf, mt = g.adjoint_pitch_run(steps, K, wx, np.zeros(steps))
    it = g.last_cg_iterations()
    g.close()
    return {"cost_ratio": mt / ms_plain, "ms_total": mt, "ms_forward_pass": mf, "ms_plain_forward": ms_plain,
            "ms_per_amplitude": mt / len(cases), "steps": steps, "checkpoint_every": K,
            "adjoint_cg_iterations_max": it, "dJ_damp_per_deg": [float(x) for x in dJ],
            "amp_deg": [c["pitch_amp_deg"] for c in cases],
            "workload": "32 plates pitching U[5,30] deg about mid-chord, f 0.25, Re 500, 512x512 cells x 5 levels, "
                        f"dt 0.001, preconditioned FP64 CG to relative 1e-12, from rest at t = 1 s; J = mean drag "
                        f"over the last {steps // 2} steps; all 32 amplitude derivatives in one batched adjoint run"}


def adjoint_cost(C, steps=100, K=50):
    """Rotating cylinder (Re 150, 256x256x4, 126 points, dt .004): the discrete
    adjoint of the mean lift over the last third of the horizon w.r.t. the
    126 tangential surface velocities (seeded N(0, 0.1^2)); cost = device time
    of the whole gradient run / device time of a plain forward run."""
    m, lev, dt, re = 256, 4, 0.004, 150.0
    xb, yb = W.circle(4.0 / m, 1.0, 0.0, 0.0, npt=126)
    th = np.arctan2(yb, xb)
    u = np.random.default_rng(SEED).normal(0.0, 0.1, 126)
    vel = np.concatenate([-u * np.sin(th), u * np.cos(th)])
    p = C.make_params(m, m, dt, re, lev)
    f = C.Solver(p, (xb, yb))
    f.precompute()
    f.advance(body_vel=vel)  # the velocities stay in force for advance_n
    f.advance_n(steps, want_hist=False)
    ms_plain = f.last_ms()
    cm, cv = f.get_cholesky()
    f.close()
    g = C.Solver(p, (xb, yb))
    g.set_cholesky(cm, cv)
    wx = np.zeros(steps)
    wy = np.zeros(steps)
    wy[-steps // 3:] = 1.0 / (steps // 3)
    J, gv, mf, mt = g.adjoint_run(steps, K, vel, wx, wy)
    g.close()
    return {"cost_ratio": mt / ms_plain, "cost_ratio_vs_own_forward_pass": mt / mf, "ms_total": mt,
            "ms_forward_pass": mf, "ms_plain_forward": ms_plain, "steps": steps, "checkpoint_every": K,
            "workload": "rotating cylinder Re 150, 256x256 cells x 4 levels, 126 points, dt 0.004, "
                        f"J = mean lift over the last {steps // 3} steps, grad w.r.t. 126 tangential velocities",
            "grad_norm": float(np.linalg.norm(gv))}


def run_ours(args):
    import torch
    import ibfs_capi as C

    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist
    pk, src = peaks()
    cases = W.batch(BATCH["ncases"], seed=SEED)[:args.ncases]
    params, bodies, opts = W.solver_args(cases, C, 1)
    for o in opts:
        o.tc_tile = args.tc_tile
    t0 = time.perf_counter()
    g = C.Solver(params, bodies, opts)
    t_create = time.perf_counter() - t0
    t0 = time.perf_counter()
    g.precompute()
    t_pre = time.perf_counter() - t0
    nlev = [s["nlev"] for s in g.sizes]
    cells = W.cells_per_step(cases, nlev)
    ncase = len(cases)
    nerr = 13  # force-history horizon of the error check (part of the warm-up)

    with ClockSampler(local) as cs:
        hist_split = g.advance_n(nerr)  # warm-up steps 1..13, recorded
        st_split = {i: g.get_state(i) for i in (0, 1, 2, 3)} if ws == 1 else None
        t_end = time.time() + 5.0
        nw = nerr
        while nw < args.warmup + nerr or (cs.count() < 1 and time.time() < t_end):
            g.advance_n(1, want_hist=False)
            nw += 1
        if pg:
            pg.barrier()
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("timed")  # lets a profiler select the timed steps
        g.advance_n(args.steps, want_hist=False)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        tot_ms = g.last_ms()
        time.sleep(0.25)
    tot_ms = max_over_ranks(tot_ms, pg)
    value = aggregate(cells, args.steps, ws, tot_ms)
    ms_per_step = tot_ms / args.steps
    kern = g.kernels_per_step()

    # end to end through the public per-step call, host buffers
    sum_nf = sum(s["nf"] for s in g.sizes)
    bvel = np.zeros(sum_nf)
    row = np.zeros(g.stride)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    te = time.perf_counter()
    for _ in range(args.steps):
        g.batch_advance(bvel, out=row)
    te = time.perf_counter() - te
    te = max_over_ranks(te, pg)
    e2e = {"value": cells * args.steps * ws / te, "unit": UNIT, "h2d_bytes_per_step": 8 * sum_nf,
           "d2h_bytes_per_step": 8 * g.stride, "call": "ibfs_batch_advance", "ms_per_step": te / args.steps * 1e3}

    prof = g.profile_step()  # one more step, CUDA events around every launch
    out = None
    if rank == 0:
        roof = roofline_gemm(prof, algorithmic_transform_flops(cases, nlev), issued_tensor_flops(cases, nlev),
                             pk, src)
        step_bytes = 64.0 * cells + sum(8.0 * s["nf"] ** 2 for s in g.sizes)
        hb = step_bytes / (ms_per_step / 1e3) / 1e9
        roof_step = {"bound": "hbm", "achieved": hb, "peak": pk["hbm_gbs"], "unit": "GB/s",
                     "frac": hb / pk["hbm_gbs"], "peak_source": src,
                     "basis": "whole step: 64 B per cell-update + 8 Nf^2 B per case"}
        extras = {}
        cpu = None
        if ws == 1 and not args.no_extras:
            # batched FP64 on the same cases, same factor; force error of the split form
            p0, b0, o0 = W.solver_args(cases, C, 0)
            f = C.Solver(p0, b0, o0)
            for i in range(ncase):
                f.set_cholesky(*g.get_cholesky(i), icase=i)
            hist_f = f.advance_n(nerr)
            fx0, fy0 = force_hist(f, hist_f, ncase)
            fx1, fy1 = force_hist(g, hist_split, ncase)
            hmax, hmed, emax, emed = force_err(fx1, fy1, fx0, fy0)
            ferr = {}
            for i in st_split:
                a, b = st_split[i]["omega"], f.get_state(i)["omega"]
                ferr[str(i)] = float(np.abs(a - b).max() / np.abs(b).max())
            f.advance_n(args.warmup, want_hist=False)
            f.advance_n(5, want_hist=False)
            fms = f.last_ms() / 5
            extras["batched_fp64"] = {"value": cells / (fms / 1e3), "ms_per_step": fms,
                                      "kernels_per_step": f.kernels_per_step()}
            extras["ratio_vs_batched_fp64"] = value / extras["batched_fp64"]["value"]
            f.close()
            extras["force_err_vs_fp64"] = {"max": hmax, "median": hmed, "per_step_max": emax,
                                           "per_step_median": emed, "steps": nerr, "cases": ncase,
                                           "basis": "relative lift/drag error of each case's force history: max "
                                                    "over steps of max(|dCd|,|dCl|) / max over steps of "
                                                    "|(Cd,Cl)|; per_step_*: divided by |(Cd,Cl)| of the same "
                                                    "step; max and median over the cases; reference = the "
                                                    "batched FP64 GPU advance (within 1e-10 of the oracle)"}
            # the same batch with two correction sweeps on the Poisson solves
            p1, b1, o1 = W.solver_args(cases, C, 1)
            for o_ in o1:
                o_.poisson_sweeps = 2
            g1 = C.Solver(p1, b1, o1)
            for i in range(ncase):
                g1.set_cholesky(*g.get_cholesky(i), icase=i)
            h1 = g1.advance_n(nerr)
            h1max, h1med, e1max, e1med = force_err(*force_hist(g1, h1, ncase), fx0, fy0)
            g1.advance_n(args.warmup, want_hist=False)
            g1.advance_n(5, want_hist=False)
            ms1 = g1.last_ms() / 5
            extras["split_two_poisson_sweeps"] = {"value": cells / (ms1 / 1e3), "ms_per_step": ms1,
                                                  "force_err_max": h1max, "force_err_median": h1med,
                                                  "force_err_per_step_max": e1max,
                                                  "force_err_per_step_median": e1med,
                                                  "kernels_per_step": g1.kernels_per_step(),
                                                  "form": "split precision, two correction sweeps on the Poisson "
                                                          "solves, one on the others"}
            g1.close()
            extras["omega_err_vs_fp64"] = {"cases": ferr, "steps": nerr, "basis": "max |d omega| / max |omega|"}
            # sequential sample: cases advanced one handle at a time
            rng = np.random.default_rng(SEED + 1)
            ids = sorted(int(x) for x in rng.choice(ncase, 16, replace=False))
            sc, sms = 0, 0.0
            for i in ids:
                s = C.Solver(params[i], bodies[i], opts[i])
                s.set_cholesky(*g.get_cholesky(i))
                s.advance_n(2, want_hist=False)
                s.advance_n(3, want_hist=False)
                sms += s.last_ms() / 3
                sc += nlev[i] * cases[i]["m"] * cases[i]["n"]
                s.close()
            extras["sequential_sample"] = {"value": sc / (sms / 1e3), "cases": ids, "form": "split-precision",
                                           "basis": "sum of cells / sum of per-case device step times"}
            flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
            plain, split = plain_and_split_plate(C, torch, args.steps, args.warmup, flush)
            extras["plain_fp64"] = plain
            extras["ratio_vs_plain_fp64"] = value / plain["value"]
            extras["plate400_split"] = split
            extras["split_err_long_horizon"] = split_error_long_horizon(C)
            extras["adjoint"] = adjoint_cost(C)
            extras["pitching_batch"] = pitching_batch(C)
            extras["pitch_adjoint"] = pitch_adjoint_cost(C)
            extras["pitch_adjoint_batch"] = pitch_adjoint_batch(C)
            extras["pitch_cg_at_max_amplitude"] = pitch_cg_at_max_amplitude(C)
            cpu = cpu_sample_from_gpu(g, cases, sorted(int(x) for x in np.random.default_rng(SEED + 2).choice(
                ncase, 6, replace=False)), args.cpu_steps)
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16x3+f64",
            "data": "synthetic (seeded cases of the named shapes; no dataset)",
            "config": batch_config(ncase, cells), "form": "batched split-precision",
            "parallelism": "replicas" if ws > 1 else "single GPU", "create_s": t_create, "precompute_s": t_pre,
            "roofline": roof, "roofline_step_hbm": roof_step, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": kern * args.steps, "kernels_per_step": kern, "profile_step": prof,
            "gemm_tiles": {name: g.gemm_tiles().count(cfg) for cfg, name in
                           ((1, "128x128/K64/2 stages"), (2, "128x256/K32/2 stages"), (3, "128x128/K32/4 stages"),
                            (4, "256x256 CTA pair/K64/2 stages"))},
            "clocks": cs.summary(), "impl": "ours",
        }
        out.update(extras)
        print(json.dumps(out), flush=True)
    g.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return out


def run_single(args):
    """--form plain / precision: the 400x400x5 plate alone (diagnostic form)."""
    import torch
    import ibfs_capi as C
    pk, src = peaks()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    plain, split = plain_and_split_plate(C, torch, args.steps, args.warmup, flush)
    d = plain if args.form == "plain" else split
    out = {"metric": METRIC, "value": d["value"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": d["ms_per_step"], "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64" if args.form == "plain" else "bf16x3+f64",
           "data": "synthetic (seeded geometry of the named config; no dataset)",
           "config": {"workload": PLATE["workload"], "form": d["form"], "l2": d["l2"] if "l2" in d else
                      "flushed between timed steps (256 MB write)"},
           "plain_fp64": plain, "plate400_split": split, "impl": "ours",
           "gpu_launches": d["kernels_per_step"] * args.steps}
    print(json.dumps(out), flush=True)


def _ref_worker(a):
    i, steps, warmup = a
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    c = W.batch(BATCH["ncases"], seed=SEED)[i]
    oc = O.Case(O.make_params(c["m"], c["n"], c["dt"], c["re"], c["levels"]), c["xb"], c["yb"])
    for _ in range(warmup):
        oc.advance()  # the first step runs preprocess (untimed), as advance does at itime==1
    t0 = time.perf_counter()
    for _ in range(steps):
        oc.advance()
    return time.perf_counter() - t0, oc.nlev * c["m"] * c["n"] * steps


def batch_config(ncases, cells):
    """The `config` of the batched headline, the same for both arms."""
    return dict(BATCH, ncases=ncases, cells_per_step=cells,
                l2="the batch state (~9 GB resident on the GPU) exceeds the 126 MB L2; no flush")


def run_reference(args):
    """The reference arm: the CPU restatement of the reference's advance (the
    oracle, a port: the Fortran+FFTW reference cannot be built here) on the
    host cores, on the same 256-case batch and the same number of timed steps
    as the GPU arm. Every (grid size, level count) stratum of the batch is
    represented by one of its cases (a plate: the step's cost depends on the
    grid, not on the body, and a plate's preprocess is the cheapest), run in
    its own process after W warm-up steps (the first runs preprocess,
    untimed), K timed steps each. The batch's throughput on P cores is the
    batch's cell-updates over its estimated wall time, sum over strata of
    (cases in stratum) x (measured time of its representative) / P: the
    256 independent cases spread over P cores."""
    ws, rank, local = dist_setup()
    if rank != 0:
        return None
    import multiprocessing as mp
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.build()
    cases = W.batch(BATCH["ncases"], seed=SEED)
    ids, wts = W.stratified_sample(cases, body="plate")
    ncores = os.cpu_count() or 1
    procs = max(1, min(ncores, args.ref_procs, len(ids)))
    steps = args.steps
    warmup = max(1, args.warmup)
    ctx = mp.get_context("spawn")
    t_wall = time.perf_counter()
    with ctx.Pool(procs) as pool:
        res = pool.map(_ref_worker, [(i, steps, warmup) for i in ids], chunksize=1)
    t_wall = time.perf_counter() - t_wall
    one_core_s = sum(w * r[0] for w, r in zip(wts, res))  # the whole batch on one core
    cells = W.cells_per_step(cases, [c["levels"] for c in cases])
    batch_s = one_core_s / procs
    value = cells * steps / batch_s
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": steps, "warmup": args.warmup,
        "ms_per_step": batch_s / steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded cases of the named shapes; no dataset)",
        "config": batch_config(len(cases), cells),
        "form": "CPU restatement of the reference's advance (oracle port), one case per process",
        "parallelism": f"{procs} host processes",
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": "port",
                         "sample": f"one plate case per (m, L) stratum of the 256-case batch ({len(ids)} strata, "
                                   f"ids {ids}), each {steps} timed steps after {warmup} warm-up steps (the first "
                                   f"runs the Cholesky preprocess, untimed), one process per case on {procs} "
                                   f"cores; batch time = sum over strata of cases x representative time / "
                                   f"{procs}; wall {t_wall:.0f} s; the Fortran+FFTW reference cannot be built "
                                   f"here, so this is the oracle port (own FFT DST-I)"},
        "strata": [{"id": i, "m": cases[i]["m"], "levels": cases[i]["levels"], "cases_in_stratum": w,
                    "s": r[0]} for i, w, r in zip(ids, wts, res)],
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
    ap.add_argument("--form", default="batch", choices=["batch", "plain", "precision"])
    ap.add_argument("--cpu-steps", type=int, default=40)
    ap.add_argument("--ncases", type=int, default=256,
                    help="first N cases of the seeded batch (a smaller case for profiler captures)")
    ap.add_argument("--no-extras", action="store_true",
                    help="headline batch measurement only (no FP64 / plate / adjoint / CPU legs)")
    ap.add_argument("--ref-procs", type=int, default=128)
    ap.add_argument("--tc-tile", type=int, default=0, choices=[0, 1, 2, 3, 4],
                    help="tensor-core GEMM tile configuration of the batched form (0: the measured autotuner)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.form == "batch":
        run_ours(args)
    else:
        run_single(args)


if __name__ == "__main__":
    main()
