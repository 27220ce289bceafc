#!/usr/bin/env python
"""Benchmark of the B200 FVT time step (SToRM solverFVT) -- one JSON line.

Workload: the 2,000,000-triangle transient meander (seeded jittered-lattice Delaunay
mesh, sloped bed + Gaussian random field, Manning n ~ U[0.02,0.06], ~30% dry cells,
Q = 200 m^3/s, Roe flux, LSQ + Barth-Jespersen, SSP-RK3 with the CFL dt reduction),
FP64.  One "step" is one iteration of solverFVT's main loop: three RK stages over the
whole mesh plus friction and the stop/mass reductions.  The metric is cell-stage
updates/s = n_cells * rkorder * steps / time.

Arms:
  --impl ours       (default) the CUDA library; `value` is device time of the K timed
                    iterations (graph replays, state resident in HBM, CUDA events on
                    the library's stream, max over ranks); `e2e` goes through the C-ABI
                    with host buffers: set_state (H2D), K x storm_fvt_step(1) each
                    returning its scalars (D2H), get_state (D2H), host wall clock.
  --impl reference  the reference algorithm on the host CPU cores: the FP64 oracle
                    port (the Fortran reference has no compiler on these machines),
                    all host threads, same mesh and metric.

Multi-GPU (one rank per GPU): `--gpus N` outside a torchrun environment re-launches
this script under torch.distributed.run with N local ranks (127.0.0.1 rendezvous).
On the single-mesh workloads every rank advances its own copy of the scenario
(replicas: independent units, no collective on the data path): weak scaling.  On
`--config batch` the ensemble's members are shared over the ranks by cell count.
`--dist-check` brings the ranks up on the gloo backend and reports them, with no GPU
work (a CPU check of the launch path).
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

import numpy as np  # noqa: E402

from storm_b200 import scenarios  # noqa: E402

METRIC = "cell-stage updates/s (FVT time step, 2M-triangle meander)"
# DRAM bytes (read + write) per cell-stage of one iteration's kernels (every stage
# kernel, k_fric and k_final), from one ncu capture of three whole iterations on the
# 500k-cell meander (dram__bytes_read.sum + dram__bytes_write.sum); traffic grows in
# proportion to the cells, so it is scaled to the workload's mesh.
NCU_DRAM_BYTES_PER_CELL_STAGE = {("meander", "phases"): 648.3}
UNIT = "cell-stage updates/s"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "source": "fallback"}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        d["source"] = "measured"
        return d
    return dict(PEAKS_FALLBACK)


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.f = None

    def __enter__(self):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        try:
            self.f.flush()
            rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        except OSError:
            rows = []
        finally:
            try:
                os.unlink(self.f.name)
            except OSError:
                pass
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except ValueError:
                continue
            for n, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def build_workload(args):
    if args.config == "meander":
        sc = scenarios.meander(n_target=args.cells)
    elif args.config == "dambreak":
        sc = scenarios.dambreak(n_target=args.cells)
    else:
        sc = scenarios.channel()
    return sc


def mesh_ratios(sc):
    from storm_b200 import fvt
    t0 = time.perf_counter()
    pm = fvt.build_mesh(sc.problem)
    mesh_ratios.build_s = time.perf_counter() - t0
    m = pm.mesh
    return pm, m.n_elems, m.n_edges, m.n_pts


def run_cpu(sc, steps, threads, warmup=0):
    """The reference algorithm (oracle port) on the host; returns (updates/s, seconds)."""
    from oracle.oracle import Oracle
    o = Oracle(sc.problem, sc.options, threads=threads)
    o.set_state(sc.h0, sc.u0, sc.v0)
    if warmup:
        o.step(warmup)
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    return sc.n_elems * sc.options.rkorder * steps / dt, dt


def run_batch(args, rank, world, local):
    """Batched steady ensemble: the --batch-n members are shared over the ranks by
    cell count (longest first onto the least-loaded rank; no data-path collective),
    each rank runs its share in one handle (one launch per kernel for all of its
    meshes), mixed precision, autotuned block shapes, to RMS dh < 1e-6 or --istop.
    Reports the whole-job cell-stage rate (cell-stages of all ranks / the slowest
    rank's device time) and the iterations / device time to steady of the members
    (cold start)."""
    import torch
    from storm_b200 import abi, build, fvt, shard
    build.build()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    params = scenarios.batch_channel_params(args.batch_n, args.batch_lo, args.batch_hi, seed=4)
    sizes = [p["n_cells"] for p in params]
    mine = shard.lpt_shards(sizes, world)[rank]
    scs = scenarios.batch_channels(args.batch_n, args.batch_lo, args.batch_hi, seed=4, only=mine,
                                   opt_limiter=args.batch_limiter, precision=abi.PREC_MIXED, device=local)
    pms = [fvt.build_mesh(sc.problem) for sc in scs]
    b = fvt.BatchSolver(pms, scs[0].options, keep=pms)
    for i, sc in enumerate(scs):
        b.set_scenario_state(i, sc.h0, sc.u0, sc.v0)
    tuned = b.autotune(iters=2)
    torch.cuda.synchronize()
    chunk, done, t_ms = 64, 0, 0.0
    conv_at = [None] * len(scs)
    launches0 = b.kernel_launches()
    stats = []
    with ClockSampler(local) as clk:
        while done < args.istop:
            n = min(chunk, args.istop - done)
            b.step(n)
            t_ms += b.last_timing()["step_ms"]
            done += n
            stats = [b.scenario_stats(i) for i in range(len(scs))]
            for i, st in enumerate(stats):
                if st["converged"] and conv_at[i] is None:
                    conv_at[i] = t_ms
            if all(st["converged"] for st in stats):
                break
    iters = np.array([st["iter"] for st in stats])
    cells = np.array([sc.n_elems for sc in scs])
    conv = np.array([c is not None for c in conv_at])
    tts = np.array([c if c is not None else np.nan for c in conv_at])
    local_res = {"cell_stages": float(np.sum(iters * cells) * 3), "device_ms": t_ms, "scenarios": len(scs),
                 "converged": int(conv.sum())}
    tot = shard.combine(local_res, dist)
    out = {
        "metric": "cell-stage updates/s (batched steady ensemble) and time-to-steady per scenario",
        "value": tot["cell_stages"] / (tot["device_ms"] / 1e3), "unit": UNIT, "n_gpus": world,
        "steps": int(iters.max()), "warmup": 0, "ms_per_step": t_ms / max(1, int(iters.max())),
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32/f64 mixed",
        "data": "synthetic (seeded generator)",
        "config": {"workload": f"batch-{args.batch_n}x[{args.batch_lo},{args.batch_hi}]",
                   "cells": int(sum(sizes)), "scenarios": args.batch_n, "rstop": 1e-6, "istop": args.istop,
                   "limiter": {0: "first order (opt 0)", 1: "LSQ (opt 1)", 2: "LSQ + BJ (opt 2)"}[args.batch_limiter],
                   "block_sizes_rank0": tuned, "parallelism": f"scenario shards x{world}",
                   "stage_path_rank0": {0: "phases", 1: "fused", 2: "fused-node-kernel"}[b.stage_path()],
                   "shard_imbalance": shard.imbalance(sizes, shard.lpt_shards(sizes, world))},
        "time_to_steady_rank0": {"converged": int(conv.sum()), "of": len(scs),
                                 "iterations_median": float(np.median(iters[conv])) if conv.any() else None,
                                 "iterations_max": int(iters[conv].max()) if conv.any() else None,
                                 "device_ms_median": float(np.nanmedian(tts)) if conv.any() else None,
                                 "device_ms_all": float(t_ms),
                                 "device_ms_per_scenario": float(t_ms) / len(scs),
                                 "cold_start": "still water, flat at the outlet level (raised to give the inlet h_n)"},
        "converged_all_ranks": tot["converged"],
        "gpu_launches": b.kernel_launches() - launches0,
        "clocks": clk.summary(),
    }
    if "per_rank_ms" in tot:
        out["per_rank_device_ms"] = tot["per_rank_ms"]
    b.close()
    if dist is not None:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))
    return 0


def run_steady_channel(args, rank, world, local):
    """Time to steady state on the 8,000-cell channel (100 m x 10 m, HLL, LSQ + BJ,
    SSP-RK3, CFL 0.9, RMS dh < 1e-8 or --istop iterations): the whole run on the GPU
    in FP64 and in mixed precision (device time of the graph replays and wall time
    through the C-ABI), against the oracle port on the host cores, timed on a bounded
    sample of the same iterations and extrapolated per iteration."""
    import torch
    from storm_b200 import abi, build, fvt
    build.build()
    torch.cuda.set_device(local)
    res = {}
    h64 = None
    for prec in ("fp64", "mixed"):
        sc = scenarios.channel()
        sc.options.device = local
        sc.options.precision = abi.PREC_MIXED if prec == "mixed" else abi.PREC_FP64
        pm = fvt.build_mesh(sc.problem)
        solver = fvt.Solver(pm, sc.options, keep=pm)
        solver.set_state(sc.h0, sc.u0, sc.v0)
        solver.step(1)
        solver.set_state(sc.h0, sc.u0, sc.v0)  # same start after the warm-up launch
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st = solver.step(args.istop)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        dev_ms = solver.last_timing()["step_ms"]
        res[prec] = {"iterations": st["iter"], "converged": bool(st["converged"]), "rms_dh": st["rms_dh"],
                     "device_s": dev_ms / 1e3, "wall_s": wall, "ms_per_iteration": dev_ms / max(1, st["iter"]),
                     "cqin": st["cqin3"][0], "cqout": st["cqout3"][0]}
        if prec == "fp64":
            h64 = solver.state()["h"]
        else:
            res[prec]["depth_max_abs_vs_fp64_m"] = float(np.abs(solver.state()["h"] - h64).max())
        solver.close()
    out = {"metric": "time to steady state (8,000-cell channel)", "value": res["fp64"]["wall_s"], "unit": "s",
           "higher_is_better": False, "n_gpus": 1, "dtype": "f64", "data": "synthetic (seeded generator)",
           "config": {"workload": "channel-8000", "rstop": 1e-8, "istop": args.istop, "flux": "HLL",
                      "limiter": "LSQ + BJ", "rk": 3, "cfl": 0.9}, "gpu": res}
    if not args.no_cpu_baseline:
        threads = len(os.sched_getaffinity(0)) or 1
        sc = scenarios.channel()
        n = max(1, min(args.istop, args.cpu_steps))
        for th, key in ((1, "cpu_1_thread"), (threads, "cpu_all_threads")):
            _, secs = run_cpu(sc, n, th)
            per_it = secs / n
            out[key] = {"cores": th, "kind": "port", "sample_iterations": n, "s_per_iteration": per_it,
                        "extrapolated_s": per_it * res["fp64"]["iterations"]}
    print(json.dumps(out))
    return 0


def run_gnn(args, rank, world, local):
    """Throughput of the warm-start network's tcgen05 kernels on a synthetic union of
    channel meshes of --cells cells: one inference forward pass and one training step
    (forward, loss, backward, Adam), CUDA events on the stream, against the measured
    dense bf16 tensor peak (the MLP products are the tensor-bound part)."""
    import torch
    from storm_b200 import build, fvt, gnn
    build.build()
    torch.cuda.set_device(local)
    dev = torch.device(f"cuda:{local}")
    rng = np.random.default_rng(0)
    nb, xn, xe, total = [], [], [], 0
    while total < args.cells:
        sc = scenarios.channel(nx=500, ny=50, seed=len(nb))
        mn = fvt.build_mesh(sc.problem).numpy()
        T = mn["n_elems"]
        nb.append(gnn.neighbour_table(mn))
        xn.append(rng.normal(size=(T, gnn.IN_NODE)).astype(np.float32))
        xe.append(rng.normal(size=(3, T, gnn.IN_EDGE)).astype(np.float32))
        total += T
    g = gnn.build_graph_fast(nb, xn, xe)
    dg = gnn.DeviceGraph(g, dev)
    net = gnn.WarmStartNet(device=dev, seed=1)
    target = torch.zeros((g.Tp, 3), dtype=torch.float32, device=dev)
    w = torch.from_numpy((np.arange(g.Tp) < g.T).astype(np.float32)).to(dev)

    def fwd_flops():
        f = 0
        for s in net.specs:
            rows = 3 * g.Tp if s.name.startswith(("edge", "enc_edge")) else g.Tp
            f += 2 * rows * (s.k_in * gnn.HID + gnn.HID * s.n_out)
        return f

    def train_flops():
        f = 0
        for s in net.specs:
            rows = 3 * g.Tp if s.name.startswith(("edge", "enc_edge")) else g.Tp
            f += 2 * rows * (s.k_in * gnn.HID + gnn.HID * s.n_out)          # forward
            f += 2 * rows * gnn.HID * s.n_out                                # dy W2
            if not s.name.startswith("enc"):
                f += 2 * rows * gnn.HID * s.k_in                             # dz1 W1
            f += 2 * rows * (s.k_in * gnn.HID + gnn.HID * s.n_out)          # dW1, dW2
        return f

    def timed(fn, n):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(n):
            fn()
        e1.record()
        torch.cuda.synchronize()
        net._check_err()
        return e0.elapsed_time(e1) / n

    def train_step():
        y = net.forward(dg, save=True)
        dy, _ = net.mse(y, target, w, 3.0 * g.T)
        net.backward(dy)
        net.adam_step(1e-4)

    n = max(1, min(args.steps, 20))
    l0 = gnn.kernel_launches()
    ms_fwd = timed(lambda: net.forward(dg, save=False), n)
    ms_train = timed(train_step, n)
    launches = gnn.kernel_launches() - l0
    pk = peaks()
    peak = pk.get("bf16_tflops") or 1590.0
    ff, tf = fwd_flops(), train_flops()
    out = {"metric": "warm-start network throughput (cells/s)", "value": g.T / (ms_fwd / 1e3),
           "unit": "cells/s (inference)", "higher_is_better": True, "n_gpus": 1, "dtype": "bf16 (fp32 accumulate)",
           "data": "synthetic graph (channel meshes, random features)",
           "config": {"workload": f"gnn-{g.T}", "cells": g.T, "layers": gnn.N_LAYERS, "hidden": gnn.HID},
           "inference": {"ms": ms_fwd, "tflops": ff / (ms_fwd / 1e3) / 1e12},
           "training_step": {"ms": ms_train, "tflops": tf / (ms_train / 1e3) / 1e12,
                             "cells_per_s": g.T / (ms_train / 1e3)},
           "roofline": {"bound": "tensor", "achieved": ff / (ms_fwd / 1e3) / 1e12, "peak": peak,
                        "unit": "TFLOP/s", "frac": ff / (ms_fwd / 1e3) / 1e12 / peak, "traffic": None,
                        "kernel": "forward pass (19 fused MLP launches)", "flops_per_launch": ff,
                        "peak_source": pk["source"]},
           "gpu_launches": launches}
    print(json.dumps(out))
    return 0


def warm_start_eval(args, local) -> dict:
    """The second half of the headline metric: time to steady state per scenario of
    held-out ensemble members, the packaged warm-start network + batched mixed solver
    against the plain FP64 solver from a cold start (one scenario at a time), with the
    ablations at equal stop tests: the analytic prior alone (zero network output) and
    the batched cold start, each to RMS dh < 1e-6 and run on to 1e-8.  Members of
    20k-40k cells when that model is packaged (else 2k-8k)."""
    from storm_b200 import warmstart
    models = os.path.join(ROOT, "storm_b200", "models")
    band = None
    for name, lo, hi in (("warmstart_channels_20k-40k.npz", 20_000, 40_000), ("warmstart_channels.npz", 2000, 8000)):
        if os.path.exists(os.path.join(models, name)):
            band = (os.path.join(models, name), lo, hi)
            break
    if band is None:
        return {"unavailable": "no trained model in the package"}
    model, lo, hi = band
    n = args.warm_eval if lo < 20_000 else min(args.warm_eval, 32)
    net, norm = warmstart.load_model(model, device=f"cuda:{local}")
    ev = warmstart.evaluate(net, norm, eval_n=n, lo=lo, hi=hi, istop=60000 if lo >= 20_000 else 40000,
                            plain_n=min(4, n), device=local, reference=True, warm_rstops=(1e-8,))

    def at(name, rs):
        r = ev[f"{name}_rstop_{rs:g}"]
        return {"s_per_scenario": r["wall_s_per_scenario_incl_preparation"],
                "speedup_vs_plain_fp64_cold": r["speedup_per_scenario_vs_plain_fp64_single_cold"],
                "iters_mean": r["iters_mean"], "converged": r["converged"],
                "depth_err_vs_steady_max_m": r["depth_err_vs_steady_max_m"], "within_1cm": r["within_1cm"]}
    return {
        "scenarios": n, "cells": f"{lo}-{hi} per scenario", "model": os.path.basename(model), "rstop": 1e-6,
        "plain_fp64_cold_s_per_scenario": ev["plain_fp64_single"]["wall_s_mean"],
        "warm_batched_mixed_s_per_scenario": ev["warm_batched_wall_s_per_scenario_incl_network"],
        "speedup_vs_plain_fp64_cold": ev["speedup_per_scenario_vs_plain_fp64_single_cold"],
        "iters_mean": {"cold": ev["cold_mixed"]["iters_mean"], "prior": ev["prior_mixed"]["iters_mean"],
                       "warm": ev["warm_mixed"]["iters_mean"]},
        "network_vs_prior_iters": ev["network_vs_prior_iters"],
        "batched_device_ms_per_scenario": {"cold_fp64": ev["cold_fp64"]["device_ms_per_scenario"],
                                           "cold_mixed": ev["cold_mixed"]["device_ms_per_scenario"],
                                           "prior_mixed": ev["prior_mixed"]["device_ms_per_scenario"],
                                           "warm_mixed": ev["warm_mixed"]["device_ms_per_scenario"]},
        # depth errors against the steady state (FP64 run on from the cold result to 1e-10)
        "depth_err_vs_steady_max_m": {k: ev["depth_err_vs_steady_max_m"][k] for k in ("warm_mixed", "cold_fp64")},
        "within_1cm": ev["within_1cm"],
        # each start against the plain FP64 cold run's own result at the same 1e-6 stop
        "depth_diff_vs_cold_fp64_same_stop": ev["depth_diff_vs_cold_fp64_same_stop"],
        # the same tighter stop test from the network, the prior alone and the cold start
        "to_1e-8": {"warm_mixed": at("warm_mixed", 1e-8), "prior_mixed": at("prior_mixed", 1e-8),
                    "cold_mixed": at("cold_mixed", 1e-8)},
    }


def run_dambreak_trajectory(args, local) -> int:
    """Config 3 in full: the circular dam break (Rusanov, Manning n = 0.025) run to
    60 s simulated in FP64 and in mixed precision side by side, one iteration at a
    time, with the mixed state compared to the FP64 state after every iteration
    (--traj-every): depth, unit discharge (hu, hv) and total mass.  Each precision
    takes its own CFL dt, so the simulated times drift apart slightly; that drift is
    reported with the errors."""
    import torch
    from storm_b200 import abi, build, fvt
    build.build()
    torch.cuda.set_device(local)
    sc = scenarios.dambreak(n_target=args.cells)
    sc.options.device = local
    t_end = float(sc.info.get("t_end", 60.0))
    pm = fvt.build_mesh(sc.problem)
    solvers = {}
    for prec in ("fp64", "mixed"):
        o = abi.Options.from_buffer_copy(sc.options)
        o.precision = abi.PREC_MIXED if prec == "mixed" else abi.PREC_FP64
        g = fvt.Solver(pm, o, keep=pm)
        g.set_state(sc.h0, sc.u0, sc.v0)
        solvers[prec] = g
    a, b = solvers["fp64"], solvers["mixed"]
    m0 = None
    rows, worst = [], {"depth_max_abs_m": 0.0, "unit_discharge_max_abs_m2s": 0.0, "mass_rel": 0.0,
                       "stime_diff_s": 0.0}
    dev_ms = {"fp64": 0.0, "mixed": 0.0}
    it = 0
    t0 = time.perf_counter()
    while True:
        sa, sb = a.step(1), b.step(1)
        dev_ms["fp64"] += a.last_timing()["step_ms"]
        dev_ms["mixed"] += b.last_timing()["step_ms"]
        it += 1
        if m0 is None:
            m0 = sa["tmass"]
        mass_rel = abs(sb["tmass"] - sa["tmass"]) / sa["tmass"]
        worst["mass_rel"] = max(worst["mass_rel"], mass_rel)
        worst["stime_diff_s"] = max(worst["stime_diff_s"], abs(sb["stime"] - sa["stime"]))
        done = sa["stime"] >= t_end or it >= args.istop
        if it % args.traj_every == 0 or done:
            xa, xb = a.state(), b.state()
            dh = np.abs(xa["h"] - xb["h"])
            dq = max(np.abs(xa["h"] * xa["u"] - xb["h"] * xb["u"]).max(),
                     np.abs(xa["h"] * xa["v"] - xb["h"] * xb["v"]).max())
            worst["depth_max_abs_m"] = max(worst["depth_max_abs_m"], float(dh.max()))
            worst["unit_discharge_max_abs_m2s"] = max(worst["unit_discharge_max_abs_m2s"], float(dq))
            if it % max(1, args.traj_every * 100) == 0 or done:
                rows.append({"iter": it, "stime_fp64": sa["stime"], "stime_mixed": sb["stime"],
                             "depth_max_abs_m": float(dh.max()), "depth_rms_m": float(np.sqrt(np.mean(dh * dh))),
                             "unit_discharge_max_abs_m2s": float(dq), "mass_rel": mass_rel,
                             "mass_drift_fp64": (sa["tmass"] - m0) / m0,
                             "wet_cells_fp64": int((xa["h"] >= sc.options.h_dry).sum())})
        if done:
            break
    wall = time.perf_counter() - t0
    out = {"metric": "config 3: mixed precision vs FP64 along a 60 s dam break, compared every iteration",
           "value": worst["depth_max_abs_m"], "unit": "m (max |h_mixed - h_fp64| over all iterations)",
           "higher_is_better": False, "n_gpus": 1, "data": "synthetic (seeded generator)",
           "config": {"workload": f"dambreak-{sc.n_elems}", "cells": sc.n_elems, "t_end_s": t_end,
                      "flux": "Rusanov", "manning": 0.025, "compare_every": args.traj_every},
           "iterations": it, "worst_over_trajectory": worst,
           "device_ms_per_iteration": {k: v / it for k, v in dev_ms.items()},
           "cell_stage_per_s": {k: sc.n_elems * 3 * it / (v / 1e3) for k, v in dev_ms.items()},
           "wall_s_including_comparisons": wall, "trajectory": rows}
    for g in solvers.values():
        g.close()
    print(json.dumps(out))
    return 0


def run_parts(args, rank, world, local) -> int:
    """`--parts P`: the meander (or dam break) as P linked parts of one handle on this
    GPU (storm_b200/partition.py) against the undivided mesh, K timed iterations of
    each; cell-stage updates count owned cells only, so the halo's redundant work and
    the exchange kernels show as the difference.  Also checks the final states bit for
    bit."""
    import torch
    from storm_b200 import build, fvt, partition
    build.build()
    torch.cuda.set_device(local)
    sc = build_workload(args)
    opt = sc.options
    opt.device = local
    t0 = time.perf_counter()
    ps = partition.PartitionedSolver(sc.problem, opt, args.parts)
    setup_s = time.perf_counter() - t0
    pm = fvt.build_mesh(sc.problem)
    whole = fvt.Solver(pm, opt, keep=pm)
    res = {}
    for name, s in (("undivided", whole), ("parts", ps)):
        s.set_state(sc.h0, sc.u0, sc.v0)
        s.step(args.warmup)
        torch.cuda.synchronize()
        s.step(args.steps)
        tm = (s.batch if name == "parts" else s).last_timing()
        res[name] = {"ms_per_step": tm["step_ms"] / args.steps,
                     "value": sc.n_elems * opt.rkorder * args.steps / (tm["step_ms"] / 1e3)}
    a, b = whole.state(), ps.state()
    same = all(np.array_equal(a[k].view(np.uint64), b[k].view(np.uint64)) for k in ("h", "u", "v"))
    halo = sum(int((~P.owned).sum()) for P in ps.parts)
    line = {"metric": f"cell-stage updates/s (FVT time step, {args.config}, {args.parts} linked parts on one GPU)",
            "value": res["parts"]["value"], "unit": "cell-stage updates/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": res["parts"]["ms_per_step"], "higher_is_better": True,
            "dtype": "f64" if opt.precision == 0 else "mixed", "data": "synthetic",
            "config": {"workload": f"{args.config}-{sc.n_elems}", "parts": args.parts,
                       "halo_cells": halo, "halo_fraction": halo / sc.n_elems},
            "undivided": res["undivided"], "bitwise_equal_to_undivided": bool(same),
            "partition_setup_s": setup_s}
    print(json.dumps(line), flush=True)
    ps.close()
    whole.close()
    return 0


def workload_config(args, T, E, N, rkorder, flux, world, dry_fraction):
    """The `config` object of the JSON line, the same keys in both arms."""
    return {"workload": f"{args.config}-{T}", "cells": T, "edges": E, "nodes": N, "rkorder": rkorder,
            "flux": int(flux), "precision": args.precision, "parallelism": f"replicas x{world}",
            "l2": "working set > L2 (inputs larger than the 126 MB L2)", "dry_fraction": dry_fraction}


def spawn_ranks(n: int) -> int:
    """Re-launch this script with the same arguments as n local ranks under
    torch.distributed.run (rendezvous on 127.0.0.1, a free port); returns its status."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", f"--master-port={port}", os.path.abspath(__file__), *sys.argv[1:]]
    return subprocess.call(cmd)


def dist_check(args, rank, world) -> int:
    """Bring the ranks up on gloo (no GPU), sum one value over them and report."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    if world > 1:
        dist.init_process_group("gloo", timeout=timedelta(seconds=60))
        t = torch.ones(1, dtype=torch.float64)
        dist.all_reduce(t)
        seen = int(t.item())
        dist.destroy_process_group()
    else:
        seen = 1
    if rank == 0:
        print(json.dumps({"metric": "launch check (no GPU work)", "dist_check": True, "n_gpus": world,
                          "ranks_seen": seen, "backend": "gloo" if world > 1 else None}))
    return 0 if seen == world else 1


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, world, local


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=["meander", "dambreak", "channel", "batch", "steady-channel", "gnn"], default="meander")
    ap.add_argument("--batch-n", type=int, default=256, help="scenarios of the batched steady ensemble")
    ap.add_argument("--batch-lo", type=int, default=20_000)
    ap.add_argument("--batch-hi", type=int, default=400_000)
    ap.add_argument("--istop", type=int, default=20_000, help="iteration cap of the steady runs")
    ap.add_argument("--batch-limiter", type=int, default=0, choices=(0, 1, 2),
                    help="opt_limiter of the steady ensemble (0: the only option whose RMS residual "
                         "reaches 1e-6 on these channels; BJ stalls near 3e-5)")
    ap.add_argument("--cells", type=int, default=2_000_000)
    ap.add_argument("--cpu-steps", type=int, default=3, help="oracle iterations timed for cpu_baseline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--autotune", action="store_true",
                    help="run the library's autotuner (stage kernels, block sizes) before timing")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64",
                    help="arithmetic of the headline run")
    ap.add_argument("--no-mixed", action="store_true", help="skip the secondary mixed-precision run")
    ap.add_argument("--cpu-budget-s", type=float, default=60.0, help="CPU seconds of the reference arm")
    ap.add_argument("--warm-eval", type=int, default=64,
                    help="held-out scenarios of the warm- vs cold-start time-to-steady, one batch (0: skip)")
    ap.add_argument("--e2e-steps", type=int, default=200, help="iterations of the end-to-end pass")
    ap.add_argument("--kt-steps", type=int, default=5, help="iterations of the per-kernel timing pass")
    ap.add_argument("--parts", type=int, default=1,
                    help="run the mesh as this many linked parts on one GPU (domain decomposition)")
    ap.add_argument("--stage-path", choices=["phases", "fused", "fused-node-kernel"], default="phases",
                    help="stage kernels of the timed runs: the phase kernels (the library's default), the fused "
                         "tile kernel, or the fused kernel with the vertex depths by k_node")
    ap.add_argument("--ab-steps", type=int, default=200,
                    help="iterations of the other stage path, timed in the same run (0: skip)")
    ap.add_argument("--trajectory", action="store_true",
                    help="--config dambreak: run 60 s simulated in FP64 and mixed, compare every iteration")
    ap.add_argument("--traj-every", type=int, default=1, help="iterations between full-state comparisons")
    ap.add_argument("--dist-check", action="store_true",
                    help="bring up --gpus ranks on gloo and report them (no GPU work)")
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return spawn_ranks(args.gpus)
    rank, world, local = dist_env()
    if args.dist_check:
        return dist_check(args, rank, world)

    if args.impl == "reference":
        if rank != 0:
            return 0
        threads = len(os.sched_getaffinity(0)) or 1
        sc = build_workload(args)
        from oracle import oracle as _o
        _o.build()
        # each timed step is one full iteration of the workload on all host threads; the
        # number of timed iterations is capped so the arm ends within about a minute
        from oracle.oracle import Oracle
        o = Oracle(sc.problem, sc.options, threads=threads)
        om = o.mesh()
        ref_config = workload_config(args, sc.n_elems, om.n_edges, om.n_pts, sc.options.rkorder, sc.options.flux,
                                     world, sc.info.get("dry_fraction"))
        o.set_state(sc.h0, sc.u0, sc.v0)
        t0 = time.perf_counter()
        o.step(max(1, min(args.warmup, 2)))
        t_iter = (time.perf_counter() - t0) / max(1, min(args.warmup, 2))
        n_timed = int(max(1, min(args.steps, round(args.cpu_budget_s / max(t_iter, 1e-6)))))
        t0 = time.perf_counter()
        o.step(n_timed)
        secs = time.perf_counter() - t0
        val = sc.n_elems * sc.options.rkorder * n_timed / secs
        out = {
            "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / n_timed,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator)",
            "config": ref_config, "host_threads": threads,
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{n_timed} of the {args.steps} requested iterations of the "
                                       f"{sc.n_elems}-cell workload, timed ({secs:.1f} s)"},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(out))
        return 0

    if args.config == "batch":
        return run_batch(args, rank, world, local)
    if args.config == "gnn":
        if rank != 0:
            return 0
        return run_gnn(args, rank, world, local)
    if args.config == "steady-channel":
        if rank != 0:
            return 0
        return run_steady_channel(args, rank, world, local)
    if args.parts > 1:
        if rank != 0:
            return 0
        return run_parts(args, rank, world, local)
    if args.trajectory:
        if rank != 0:
            return 0
        return run_dambreak_trajectory(args, local)

    import torch
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    torch.cuda.set_device(local)

    from storm_b200 import build, fvt
    build.build()
    sc = build_workload(args)
    sc.options.device = local
    if args.precision == "mixed":
        sc.options.precision = 1
    pm, T, E, N = mesh_ratios(sc)
    K_rk = sc.options.rkorder
    t0 = time.perf_counter()
    solver = fvt.Solver(pm, sc.options, keep=pm)
    solver.set_stage_path({"phases": fvt.STAGE_PHASES, "fused": fvt.STAGE_FUSED,
                           "fused-node-kernel": fvt.STAGE_FUSED_NODE_KERNEL}[args.stage_path])
    tuned = None
    if args.autotune:  # stage path and block sizes by timing (state restored; outside the timed region)
        solver.set_state(sc.h0, sc.u0, sc.v0)
        tuned = solver.autotune(iters=3)
    path_used = {fvt.STAGE_PHASES: "phases", fvt.STAGE_FUSED: "fused",
                 fvt.STAGE_FUSED_NODE_KERNEL: "fused-node-kernel"}[solver.stage_path()]
    setup = {"mesh_build_s": mesh_ratios.build_s, "create_s": time.perf_counter() - t0,
             "what": "storm_fvt_mesh_build (topology, edges, walls, boundary arrays, LSQ and IDW set-up: "
                     "read_data + dataprepFVT, host C++) and storm_fvt_create (layout, upload, graph capture)"}

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- device-resident timed region ----
    solver.set_state(sc.h0, sc.u0, sc.v0)
    solver.step(args.warmup)
    barrier()
    launches0 = solver.kernel_launches()
    with ClockSampler(local) as clk:
        barrier()
        stats = solver.step(args.steps)
        barrier()
    ms = solver.last_timing()["step_ms"]
    gpu_launches = solver.kernel_launches() - launches0
    ref_state = solver.state() if not args.no_mixed else None
    ms_max = ms
    if dist is not None:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
    value = world * T * K_rk * args.steps / (ms_max / 1e3)

    # ---- end-to-end through the C-ABI with host buffers ----
    e2e_steps = max(1, min(args.steps, args.e2e_steps))
    barrier()
    t0 = time.perf_counter()
    solver.set_state(sc.h0, sc.u0, sc.v0)
    for _ in range(e2e_steps):
        solver.step(1)
    st = solver.state(("h", "u", "v"))  # the result: depth and velocities in element order
    barrier()
    e2e_s = time.perf_counter() - t0
    if dist is not None:
        t = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_val = world * T * K_rk * e2e_steps / e2e_s
    h2d = 3 * 8 * T / e2e_steps
    d2h = 224 + (3 * 8 * T) / e2e_steps  # StepStats per call + the final h, u, v

    # ---- secondary run in the other precision: speed and error vs this run ----
    other = None
    if not args.no_mixed:
        import ctypes
        from storm_b200 import abi
        o2 = abi.Options.from_buffer_copy(sc.options)
        o2.precision = 0 if args.precision == "mixed" else 1
        s2 = fvt.Solver(pm, o2, keep=pm)
        s2.set_state(sc.h0, sc.u0, sc.v0)
        s2.step(args.warmup)
        barrier()
        st2 = s2.step(args.steps)
        barrier()
        ms2 = s2.last_timing()["step_ms"]
        b_state = s2.state()
        a_state = ref_state
        if args.precision == "mixed":
            a_state, b_state = b_state, a_state
        hu_a, hv_a = a_state["h"] * a_state["u"], a_state["h"] * a_state["v"]
        hu_b, hv_b = b_state["h"] * b_state["u"], b_state["h"] * b_state["v"]
        qs = max(float(np.abs(hu_a).max()), float(np.abs(hv_a).max()), 1e-12)
        other = {
            "precision": "mixed" if args.precision == "fp64" else "fp64",
            "value": T * K_rk * args.steps / (ms2 / 1e3), "ms_per_step": ms2 / args.steps,
            "error_vs_fp64_after_steps": args.warmup + args.steps,
            "depth_max_abs_m": float(np.abs(a_state["h"] - b_state["h"]).max()),
            "depth_rms_m": float(np.sqrt(np.mean((a_state["h"] - b_state["h"]) ** 2))),
            "momentum_max_rel": float(max(np.abs(hu_a - hu_b).max(), np.abs(hv_a - hv_b).max()) / qs),
            "mass_rel": abs(st2["tmass"] - stats["tmass"]) / stats["tmass"],
        }
        s2.close()

    # ---- the other stage paths on the same mesh: speed and bitwise agreement ----
    ab = None
    if args.ab_steps > 0:
        n_ab = max(1, min(args.steps, args.ab_steps))
        names = {fvt.STAGE_PHASES: "phases", fvt.STAGE_FUSED: "fused",
                 fvt.STAGE_FUSED_NODE_KERNEL: "fused, vertex depths by k_node"}
        solver.set_state(sc.h0, sc.u0, sc.v0)
        solver.step(args.warmup)
        barrier()
        solver.step(n_ab)
        barrier()
        ms_this, st_this = solver.last_timing()["step_ms"], solver.state()
        ab = {"steps": n_ab, "this_path_ms_per_step": ms_this / n_ab, "others": []}
        for other_path in names:
            if other_path == solver.stage_path():
                continue
            s3 = fvt.Solver(pm, sc.options, keep=pm)
            s3.set_stage_path(other_path)
            if s3.stage_path() == other_path:
                s3.set_state(sc.h0, sc.u0, sc.v0)
                s3.step(args.warmup)
                barrier()
                s3.step(n_ab)
                barrier()
                ms3, st3 = s3.last_timing()["step_ms"], s3.state()
                same = all(np.array_equal(st_this[k].view(np.uint64), st3[k].view(np.uint64))
                           for k in ("h", "u", "v", "rku", "rkv", "hvtx"))
                ab["others"].append({"stage_kernels": names[other_path], "ms_per_step": ms3 / n_ab,
                                     "value": T * K_rk * n_ab / (ms3 / 1e3), "bitwise_equal_states": bool(same)})
            s3.close()

    # ---- per-kernel timing pass (roofline of the RK-stage kernel chain) ----
    solver.set_state(sc.h0, sc.u0, sc.v0)
    solver.set_kernel_timing(True)
    kt_steps = max(1, args.kt_steps)
    solver.step(kt_steps)
    kt = solver.kernel_times()
    solver.set_kernel_timing(False)
    stage_ms = sum(kt[k][0] for k in ("node", "grad", "bc", "eflux", "flux", "tile"))
    B = scenarios.algorithmic_bytes_per_cell_stage(T, E, N)
    pk = peaks()
    # The launch unit is one graph replay = one iteration (K stages of every kernel,
    # friction and the reductions), timed with CUDA events on the library's stream over
    # the timed region above; the per-kernel pass (serialised, one event pair per
    # launch, the boundary kernel no longer overlapped) gives the shares.
    ms_iter = ms_max / args.steps
    achieved = B * T * K_rk / (ms_iter / 1e3) / 1e9
    achieved_serial = B * T * K_rk * kt_steps / (stage_ms / 1e3) / 1e9
    iter_ms = sum(v[0] for v in kt.values())
    traffic = None
    if (args.config, path_used) in NCU_DRAM_BYTES_PER_CELL_STAGE:
        traffic = NCU_DRAM_BYTES_PER_CELL_STAGE[(args.config, path_used)] * T * K_rk
    chain = {"fused": "K x [k_node(boundary-cell vertices) -> k_grad(boundary cells) -> k_bc || k_tile, k_flux_bc]",
             "fused-node-kernel": "K x [k_node, k_grad(boundary cells) -> k_bc || k_tile, k_flux_bc]",
             "phases": "K x [k_node, k_grad, k_bc || k_eflux, k_flux, k_flux_bc]"}[path_used]
    roofline = {
        "bound": "hbm", "achieved": achieved, "peak": pk.get("hbm_gbs"), "unit": "GB/s",
        "frac": achieved / pk["hbm_gbs"], "traffic": traffic,
        "kernel": f"one iteration (CUDA graph: {chain}, k_fric, k_final)",
        "algorithmic_bytes_per_launch": B * T * K_rk, "bytes_per_cell_stage": B, "peak_source": pk["source"],
        "traffic_source": "ncu dram__bytes_read+write of three iterations' kernels on the 500k-cell "
                          "meander, per cell-stage, scaled to this mesh" if traffic else None,
        "achieved_serialised_stage_chain": achieved_serial,
        "kernel_ms_share": {k: round(v[0] / iter_ms, 4) for k, v in kt.items()},
        "stage_kernel_avg_ms": (kt["tile"][0] / max(1, kt["tile"][1]) if path_used != "phases"
                                else kt["flux"][0] / max(1, kt["flux"][1])),
    }

    metric = METRIC if args.config == "meander" else f"cell-stage updates/s (FVT time step, {args.config})"
    out = {
        "metric": metric, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32/f64 mixed",
        "data": "synthetic (seeded generator; no public dataset exists for this path)",
        "config": workload_config(args, T, E, N, K_rk, sc.options.flux, world, sc.info.get("dry_fraction")),
        "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": e2e_steps},
        "gpu_launches": gpu_launches,
        "stage_kernels": path_used,
        "block_sizes": tuned if tuned is not None else "library defaults (node 128, grad 64, eflux 64 FP64 / 128 mixed, flux 64)",
        "setup": setup,
        "roofline": roofline,
        "clocks": clk.summary(),
        "final": {"iter": stats["iter"], "tmass": stats["tmass"], "status": stats["device_status"]},
    }
    if other is not None:
        out["other_precision"] = other
    if ab is not None:
        out["other_stage_kernels"] = ab
    if rank == 0 and world == 1 and args.warm_eval > 0 and args.config == "meander":
        out["time_to_steady"] = warm_start_eval(args, local)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = len(os.sched_getaffinity(0)) or 1
        cv, secs = run_cpu(sc, args.cpu_steps, threads)
        out["cpu_baseline"] = {"value": cv, "unit": UNIT, "cores": threads, "kind": "port",
                               "sample": f"{args.cpu_steps} iterations of the same {T}-cell workload "
                                         f"({secs:.1f} s on {threads} threads)"}
    solver.close()
    if dist is not None:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
