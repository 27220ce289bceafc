"""Warm-start pipeline for steady runs: features of a scenario, solver-generated
training data, training of :class:`storm_b200.gnn.WarmStartNet` on the GPU, and the
prediction handed to the solver as its initial state.

The inputs of the network are what the Fortran host holds at the solverFVT call:
the bed (``z``, ``zvtx``), Manning's n (``cd``), the cell geometry (area, centroid),
the boundary discharge ``qin`` and stage ``hbc`` and which cells carry inflow,
outflow or wall faces.  From these the host derives, per mesh, a few descriptors
that no 8-hop message passing could see: the along-channel distance of every cell
to the outflow (a shortest path over the cell-dual graph), the channel length, mean
width and slope, and the Manning normal depth h_n = (n Q / (W sqrt(S)))^(3/5).

Targets are expressed against a depth prior d0 = max(hbc - zb, h_n) (still water
at the outlet stage, but at least the normal depth) and the unit discharge Q/W:
t = [(h - d0) / 1 m, hu / (Q/W), hv / (Q/W)].
"""
from __future__ import annotations

import dataclasses
import math
import time

import numpy as np

from . import abi, fvt, gnn


@dataclasses.dataclass
class Inputs:
    nbr: np.ndarray      # [3, T]
    x_node: np.ndarray   # [T, 64]
    x_edge: np.ndarray   # [3, T, 64]
    d0: np.ndarray       # [T] depth prior
    qw: float            # Q / W, unit discharge scale
    h_dry: float


def _boundary_cells(mn: dict, kind: str) -> np.ndarray:
    """0-based cells with a face on the inflow / outflow boundaries."""
    T = mn["n_elems"]
    if kind == "in":
        ld, nb, arr = mn["bcin_ld"], mn["n_inflowbdr"], mn["bcedgesinflow"]
    else:
        ld, nb, arr = mn["bcout_ld"], mn["n_outflowbdr"], mn["bcedgesoutflow"]
    cells = []
    edge_e = mn["edge_e"].reshape(-1, 2)
    for b in range(nb):
        col = arr[b * ld:(b + 1) * ld]
        n = int(col[0])
        for k in range(1, n + 1):
            ed = abs(int(col[k])) - 1
            e1, e2 = edge_e[ed]
            cells.append((e1 if e1 > 0 else e2) - 1)
    out = np.unique(np.array(cells, dtype=np.int64))
    return out[(out >= 0) & (out < T)]


def scenario_inputs(mn: dict, q: float, hbc: float, h_dry: float = 1e-3) -> Inputs:
    """Features of one prepared mesh (`mn` = PreparedMesh.numpy()) with inflow q and
    outlet stage hbc (water-surface elevation)."""
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import dijkstra
    T = int(mn["n_elems"])
    nbr = gnn.neighbour_table(mn)
    xc, yc = mn["tri_xc"], mn["tri_yc"]
    zb, area, n = mn["z"], mn["tri_area"], mn["cd"]
    ell = np.sqrt(area)
    cin = _boundary_cells(mn, "in")
    cout = _boundary_cells(mn, "out")
    wall = np.zeros(T, dtype=bool)
    wall[(nbr < 0).any(axis=0)] = True
    fin = np.zeros(T, dtype=bool)
    fin[cin] = True
    fout = np.zeros(T, dtype=bool)
    fout[cout] = True
    wall &= ~(fin | fout)
    # along-channel distance to the outflow over the cell-dual graph
    k, c = np.nonzero(nbr >= 0)
    s = nbr[k, c]
    w = np.hypot(xc[s] - xc[c], yc[s] - yc[c])
    G = coo_matrix((w, (c, s)), shape=(T, T)).tocsr()
    dist = dijkstra(G, directed=False, indices=cout, min_only=True)
    dist = np.where(np.isfinite(dist), dist, 0.0)
    L = float(max(dist[cin].mean() if len(cin) else dist.max(), 1.0))
    W = float(area.sum() / L)
    zin = float(zb[cin].mean()) if len(cin) else float(zb.max())
    zout = float(zb[cout].mean()) if len(cout) else float(zb.min())
    S = float(max((zin - zout) / L, 1e-5))
    nbar = float(n.mean())
    h_n = (nbar * q / (W * math.sqrt(S))) ** 0.6
    d_still = np.maximum(hbc - zb, 0.0)
    d0 = np.maximum(d_still, h_n)
    qw = q / W
    xn = np.zeros((T, gnn.IN_NODE), dtype=np.float32)
    cols = [
        (zb - hbc) / 2.0, d_still / 5.0, n * 20.0, ell / 2.0, np.full(T, q / 250.0),
        np.full(T, math.log(q / 100.0)), np.full(T, (hbc - zout) / 5.0), fin, fout, wall,
        dist / L, dist / 100.0, np.full(T, W / 50.0), np.full(T, S * 1000.0), np.full(T, h_n / 5.0),
        np.full(T, qw / h_n / 5.0), np.full(T, (hbc - zout - h_n) / 2.0), d0 / 5.0,
    ]
    for j, v in enumerate(cols):
        xn[:, j] = v
    xe = np.zeros((3, T, gnn.IN_EDGE), dtype=np.float32)
    valid = nbr >= 0
    src = np.where(valid, nbr, 0)
    dx = (xc[src] - xc[None, :]) / ell[None, :]
    dy = (yc[src] - yc[None, :]) / ell[None, :]
    dd = np.hypot(dx, dy)
    dz = (zb[src] - zb[None, :]) * 100.0
    ds = (dist[src] - dist[None, :]) / np.maximum(np.hypot(xc[src] - xc[None, :], yc[src] - yc[None, :]), 1e-9)
    for j, v in enumerate((dx, dy, dd, dz, ds, np.ones_like(dx))):
        xe[:, :, j] = np.where(valid, v, 0.0)
    return Inputs(nbr, xn, xe, d0, qw, h_dry)


def targets(inp: Inputs, h, u, v) -> np.ndarray:
    t = np.zeros((len(h), 3), dtype=np.float32)
    t[:, 0] = h - inp.d0
    t[:, 1] = h * u / inp.qw
    t[:, 2] = h * v / inp.qw
    return t


def state_from_prediction(inp: Inputs, t: np.ndarray):
    """Initial h, u, v for the solver from the network's output rows."""
    h = np.maximum(inp.d0 + t[:, 0].astype(np.float64), 0.0)
    hu = t[:, 1].astype(np.float64) * inp.qw
    hv = t[:, 2].astype(np.float64) * inp.qw
    wet = h > inp.h_dry
    u = np.where(wet, hu / np.where(wet, h, 1.0), 0.0)
    v = np.where(wet, hv / np.where(wet, h, 1.0), 0.0)
    return h, u, v


def scenario_q_hbc(sc) -> tuple[float, float]:
    return float(sc.info["q"]), float(sc.info["hbc"])


# ---- solver runs ---------------------------------------------------------------------

def run_steady_batch(scs, states=None, istop: int = 40000, chunk: int = 64, precision=abi.PREC_MIXED,
                     device: int = 0, autotune: bool = True, keep_states: bool = True, rstop=None):
    """Run scenarios together to their stop test (or istop).  `states` (optional) is a
    list of (h, u, v) initial states; default is each scenario's cold start.  Returns
    per-scenario iterations, convergence time (ms of device time from the start) and,
    with keep_states, the final h, u, v."""
    pms = [fvt.build_mesh(sc.problem) for sc in scs]
    opt = abi.default_options(**{f: getattr(scs[0].options, f) for f, _ in abi.Options._fields_
                                 if f not in ("reserved",)})
    opt.precision = precision
    opt.device = device
    if rstop is not None:
        opt.rstop = rstop
    b = fvt.BatchSolver(pms, opt, keep=pms)
    for i, sc in enumerate(scs):
        h, u, v = states[i] if states is not None else (sc.h0, sc.u0, sc.v0)
        b.set_scenario_state(i, h, u, v)
    tuned = b.autotune(iters=2) if autotune else None
    done, t_ms = 0, 0.0
    conv_ms = [None] * len(scs)
    t0 = time.perf_counter()
    stats = []
    while done < istop:
        n = min(chunk, istop - done)
        b.step(n)
        t_ms += b.last_timing()["step_ms"]
        done += n
        stats = [b.scenario_stats(i) for i in range(len(scs))]
        for i, st in enumerate(stats):
            if st["converged"] and conv_ms[i] is None:
                conv_ms[i] = t_ms
        if all(st["converged"] for st in stats):
            break
    wall = time.perf_counter() - t0
    out = {"iters": np.array([st["iter"] for st in stats]), "converged": np.array([bool(st["converged"]) for st in stats]),
           "conv_ms": np.array([c if c is not None else np.nan for c in conv_ms]), "device_ms": t_ms, "wall_s": wall,
           "rmax": np.array([st["rmax"] for st in stats]), "block_sizes": tuned,
           "stage_path": b.stage_path(), "launches": b.kernel_launches()}
    if keep_states:
        out["states"] = [b.scenario_state(i) for i in range(len(scs))]
    b.close()
    return out


# ---- training -------------------------------------------------------------------------

@dataclasses.dataclass
class Sample:
    inp: Inputs
    target: np.ndarray


@dataclasses.dataclass
class Normalizer:
    """Per-column standardisation of the node and edge inputs (fitted on the training
    set, padded columns stay zero) and of the three targets."""
    node_mean: np.ndarray
    node_std: np.ndarray
    edge_mean: np.ndarray
    edge_std: np.ndarray
    t_mean: np.ndarray
    t_std: np.ndarray

    @staticmethod
    def fit(samples) -> "Normalizer":
        xn = np.concatenate([s.inp.x_node for s in samples]).astype(np.float64)
        xe = np.concatenate([s.inp.x_edge[s.inp.nbr >= 0] for s in samples]).astype(np.float64)
        t = np.concatenate([s.target for s in samples]).astype(np.float64)

        def ms(a):
            m, sd = a.mean(axis=0), a.std(axis=0)
            used = sd > 1e-12
            return np.where(used, m, 0.0).astype(np.float32), np.where(used, sd, 1.0).astype(np.float32)
        nm, ns = ms(xn)
        em, es = ms(xe)
        tm, ts = ms(t)
        return Normalizer(nm, ns, em, es, tm, ts)

    def inputs(self, inp: Inputs) -> Inputs:
        xn = (inp.x_node - self.node_mean) / self.node_std
        xe = (inp.x_edge - self.edge_mean) / self.edge_std
        xe[inp.nbr < 0] = 0.0
        return dataclasses.replace(inp, x_node=xn.astype(np.float32), x_edge=xe.astype(np.float32))

    def target(self, t):
        return ((t - self.t_mean) / self.t_std).astype(np.float32)

    def untarget(self, y):
        return y * self.t_std + self.t_mean

    def arrays(self) -> dict:
        return {k: getattr(self, k) for k in ("node_mean", "node_std", "edge_mean", "edge_std", "t_mean", "t_std")}


def make_sample(sc, state) -> Sample:
    pm = fvt.build_mesh(sc.problem)
    q, hbc = scenario_q_hbc(sc)
    inp = scenario_inputs(pm.numpy(), q, hbc, sc.options.h_dry)
    return Sample(inp, targets(inp, state["h"], state["u"], state["v"]))


class DeviceBatch:
    def __init__(self, samples, device, norm: Normalizer):
        import torch
        inps = [norm.inputs(s.inp) for s in samples]
        g = gnn.build_graph_fast([i.nbr for i in inps], [i.x_node for i in inps], [i.x_edge for i in inps])
        self.graph = gnn.DeviceGraph(g, device)
        t = np.zeros((g.Tp, 3), dtype=np.float32)
        w = np.zeros(g.Tp, dtype=np.float32)
        for i, s in enumerate(samples):
            o = g.cell_off[i]
            t[o:o + len(s.target)] = norm.target(s.target)
            w[o:o + len(s.target)] = 1.0
        self.target = torch.from_numpy(t).to(device)
        self.w = torch.from_numpy(w).to(device)
        self.T = g.T
        self.offsets = g.cell_off


def group_samples(samples, cells_per_batch: int):
    groups, cur, n = [], [], 0
    for s in samples:
        T = len(s.target)
        if cur and n + T > cells_per_batch:
            groups.append(cur)
            cur, n = [], 0
        cur.append(s)
        n += T
    if cur:
        groups.append(cur)
    return groups


def train(net: gnn.WarmStartNet, batches, epochs: int, lr: float = 1e-3, lr_min: float = 1e-5,
          clip: float = 1.0, log=None) -> list:
    """Adam with a cosine learning-rate schedule and global-norm clipping; returns the
    mean loss of every epoch."""
    import torch
    history = []
    total_steps = epochs * len(batches)
    step = 0
    for ep in range(epochs):
        losses = []
        for bi in np.random.default_rng(ep).permutation(len(batches)):
            b = batches[bi]
            y = net.forward(b.graph, save=True)
            dy, parts = net.mse(y, b.target, b.w, 3.0 * b.T)
            net.backward(dy)
            gn = net.grad_norm()
            step += 1
            if not math.isfinite(gn):  # skip the update; the loss history shows it
                losses.append(float("nan"))
                continue
            scale = 1.0 if gn <= clip else clip / gn
            warm = min(1.0, step / max(1.0, 0.03 * total_steps))
            lr_t = warm * (lr_min + 0.5 * (lr - lr_min) * (1 + math.cos(math.pi * step / max(1, total_steps))))
            net.adam_step(lr_t, grad_scale=scale)
            losses.append(float(parts.cpu().numpy().astype(np.float64).sum()))
        torch.cuda.synchronize()
        net._check_err()
        history.append(float(np.nanmean(losses)) if np.isfinite(losses).any() else float("nan"))
        if log:
            log(f"epoch {ep}: loss {history[-1]:.5f}")
    return history


def predict(net: gnn.WarmStartNet, norm: Normalizer, samples_inputs, device, timing: dict | None = None) -> list:
    """Network output rows [T, 3] (in target units) for each Inputs (one batched
    forward pass).  With `timing`, fills host_s (normalisation, graph union, upload,
    read-back) and device_ms (the forward kernels, CUDA events)."""
    import torch
    t0 = time.perf_counter()
    inps = [norm.inputs(i) for i in samples_inputs]
    g = gnn.build_graph_fast([i.nbr for i in inps], [i.x_node for i in inps], [i.x_edge for i in inps])
    dg = gnn.DeviceGraph(g, device)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    y = net.forward(dg, save=False)
    e1.record()
    torch.cuda.synchronize()
    net._check_err()
    yn = y.cpu().numpy()
    if timing is not None:
        dev_ms = e0.elapsed_time(e1)
        timing["device_ms"] = dev_ms
        timing["host_s"] = (t1 - t0) + max(0.0, time.perf_counter() - t1 - dev_ms / 1e3)
        timing["cells"] = g.T
    return [norm.untarget(yn[g.cell_off[i]:g.cell_off[i + 1], :3]) for i in range(len(samples_inputs))]


def load_model(path, device="cuda:0"):
    """A trained network and its normaliser from an .npz written by :func:`pipeline`."""
    z = np.load(path)
    net = gnn.WarmStartNet(device=device, params=z["params"].astype(np.float32))
    norm = Normalizer(*(z[k] for k in ("node_mean", "node_std", "edge_mean", "edge_std", "t_mean", "t_std")))
    return net, norm


# ---- end-to-end: data, training, evaluation --------------------------------------------

def _member_list(n, lo, hi, seed, limiter):
    from . import scenarios
    return scenarios.batch_channels(n, lo, hi, seed=seed, opt_limiter=limiter)


def pipeline(train_n=4096, eval_n=64, lo=2000, hi=8000, gen_batch=512, istop=40000, epochs=30,
             cells_per_batch=400_000, lr=1e-3, limiter=0, device=0, seed=7, log=print, weights_out=None,
             warm_rstops=(), plain_n=8):
    """Generate `train_n` steady states with the solver (mixed precision), train the
    network on them, then run the `eval_n` held-out scenarios (seeds disjoint) to
    steady state cold in FP64, cold in mixed precision and warm in mixed precision.
    Returns a summary dict."""
    import torch
    torch.cuda.set_device(device)
    dev = torch.device(f"cuda:{device}")
    res = {"config": {"train_n": train_n, "eval_n": eval_n, "cells": [lo, hi], "istop": istop, "epochs": epochs,
                      "limiter": limiter, "rstop": 1e-6, "layers": gnn.N_LAYERS, "hidden": gnn.HID}}
    # 1. training data
    t0 = time.perf_counter()
    samples, gen_iters, gen_ms, not_conv = [], [], 0.0, 0
    for b0 in range(0, train_n, gen_batch):
        nb = min(gen_batch, train_n - b0)
        scs = _member_list(nb, lo, hi, seed=seed * 100003 + b0, limiter=limiter)
        r = run_steady_batch(scs, istop=istop, precision=abi.PREC_MIXED, device=device)
        gen_ms += r["device_ms"]
        gen_iters += r["iters"].tolist()
        for sc, st, ok in zip(scs, r["states"], r["converged"]):
            if not ok:
                not_conv += 1
                continue
            samples.append(make_sample(sc, st))
        log(f"generated {len(samples)} steady states ({not_conv} unconverged), {gen_ms / 1e3:.1f} s device")
    res["data"] = {"states": len(samples), "unconverged": not_conv, "device_s": gen_ms / 1e3,
                   "wall_s": time.perf_counter() - t0, "iters_median": float(np.median(gen_iters)),
                   "cells": int(sum(len(s.target) for s in samples))}
    # 2. training
    t1 = time.perf_counter()
    norm = Normalizer.fit(samples)
    batches = [DeviceBatch(g, dev, norm) for g in group_samples(samples, cells_per_batch)]
    net = gnn.WarmStartNet(device=dev, seed=seed)
    l0 = gnn.kernel_launches()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    hist = train(net, batches, epochs, lr=lr, log=log)
    ev1.record()
    torch.cuda.synchronize()
    res["train"] = {"loss_first": hist[0], "loss_last": hist[-1], "history": hist, "batches": len(batches),
                    "device_s": ev0.elapsed_time(ev1) / 1e3, "wall_s": time.perf_counter() - t1,
                    "kernel_launches": gnn.kernel_launches() - l0}
    if weights_out:
        np.savez(weights_out, params=net.params_numpy(), **norm.arrays())
    del batches
    # 3. evaluation on held-out scenarios
    res["eval"] = evaluate(net, norm, eval_n, lo, hi, istop, limiter, device, seed, plain_n=plain_n,
                           warm_rstops=warm_rstops)
    return res


def evaluate(net, norm, eval_n=64, lo=2000, hi=8000, istop=40000, limiter=0, device=0, seed=7,
             plain_n=8, reference=True, warm_rstops=()) -> dict:
    """Held-out scenarios (seeds disjoint from the training data) run to the stop test:
    cold FP64 and cold mixed (batched), warm mixed (batched, from the network's
    prediction), the plain FP64 solver on each scenario alone (the first `plain_n`),
    and an FP64 continuation to RMS dh < 1e-10 as the steady state the depth errors
    are measured against.  `warm_rstops` adds warm mixed runs to tighter residuals
    (time and depth error of each, and how many members end within 1 cm)."""
    import torch
    dev = torch.device(f"cuda:{device}")
    ev = _member_list(eval_n, lo, hi, seed=seed * 100003 + 99_999_989, limiter=limiter)
    inps = []
    tf = time.perf_counter()
    for sc in ev:
        pm = fvt.build_mesh(sc.problem)
        q, hbc = scenario_q_hbc(sc)
        inps.append(scenario_inputs(pm.numpy(), q, hbc, sc.options.h_dry))
    feat_s = time.perf_counter() - tf
    predict(net, norm, inps[:2], dev)  # warm-up (kernel attributes, allocator)
    tm = {}
    preds = predict(net, norm, inps, dev, timing=tm)
    infer_ms = tm["device_ms"]
    warm_states = [state_from_prediction(i, p) for i, p in zip(inps, preds)]
    # the analytic prior alone: zero network output through the same mapping
    prior_states = [state_from_prediction(i, np.zeros((len(i.d0), 3), dtype=np.float32)) for i in inps]
    cold64 = run_steady_batch(ev, istop=istop, precision=abi.PREC_FP64, device=device)
    cold_mx = run_steady_batch(ev, istop=istop, precision=abi.PREC_MIXED, device=device)
    warm_mx = run_steady_batch(ev, states=warm_states, istop=istop, precision=abi.PREC_MIXED, device=device)
    prior_mx = run_steady_batch(ev, states=prior_states, istop=istop, precision=abi.PREC_MIXED, device=device)
    # the steady state itself: FP64 run on from the cold-start result to RMS dh < 1e-10
    # (without it, depths are compared with the cold FP64 run's own stop state)
    if reference:
        ref = run_steady_batch(ev, states=[(s["h"], s["u"], s["v"]) for s in cold64["states"]],
                               istop=4 * istop, precision=abi.PREC_FP64, device=device, rstop=1e-10)
    else:
        ref = {"states": cold64["states"], "converged": cold64["converged"], "iters": cold64["iters"] * 0}

    def dmax(states, key="h"):
        return [float(np.max(np.abs((a[key] if isinstance(a, dict) else a[0]) - b["h"])))
                for a, b in zip(states, ref["states"])]
    dh_warm, dh_cold, dh_cold64 = dmax(warm_mx["states"]), dmax(cold_mx["states"]), dmax(cold64["states"])
    dh_pred = dmax(warm_states)

    def summ(r):
        return {"stage_path": {0: "phases", 1: "fused", 2: "fused-node-kernel"}.get(r.get("stage_path"), None),
                "converged": int(r["converged"].sum()), "iters_mean": float(r["iters"].mean()),
                "iters_median": float(np.median(r["iters"])), "iters_max": int(r["iters"].max()),
                "device_s_batch": r["device_ms"] / 1e3, "device_ms_per_scenario": r["device_ms"] / len(ev),
                "wall_s_batch": r["wall_s"]}

    dh_prior = dmax(prior_mx["states"])
    out = {"cold_fp64": summ(cold64), "cold_mixed": summ(cold_mx), "warm_mixed": summ(warm_mx),
           "prior_mixed": dict(summ(prior_mx), depth_err_vs_steady_max_m=max(dh_prior),
                               depth_err_vs_steady_median_m=float(np.median(dh_prior)),
                               within_1cm=int(sum(x <= 0.01 for x in dh_prior))),
           "network_vs_prior_iters": float(prior_mx["iters"].mean() / max(warm_mx["iters"].mean(), 1)),
                   "inference_ms_batch": infer_ms, "inference_host_s_batch": tm["host_s"],
                   "features_host_s_batch": feat_s,
                   "speedup_per_scenario_vs_cold_fp64": (cold64["device_ms"]) / (warm_mx["device_ms"] + infer_ms),
                   "speedup_per_scenario_vs_cold_fp64_incl_host": (cold64["wall_s"]) / (
                       warm_mx["wall_s"] + infer_ms / 1e3 + tm["host_s"] + feat_s),
                   "speedup_iters_vs_cold": float(cold_mx["iters"].mean() / max(warm_mx["iters"].mean(), 1)),
                   "steady_reference": {"rstop": 1e-10 if reference else 1e-6,
                                        "converged": int(ref["converged"].sum()),
                                        "iters_mean_beyond_1e-6": float(ref["iters"].mean())},
                   "depth_err_vs_steady_max_m": {"warm_mixed": max(dh_warm), "cold_mixed": max(dh_cold),
                                                 "cold_fp64": max(dh_cold64), "prediction": max(dh_pred)},
                   "depth_err_vs_steady_median_m": {"warm_mixed": float(np.median(dh_warm)),
                                                    "cold_mixed": float(np.median(dh_cold)),
                                                    "cold_fp64": float(np.median(dh_cold64)),
                                                    "prediction": float(np.median(dh_pred))}}
    # the same tighter stop tests from the warm start, the prior alone and the cold start
    for rs in warm_rstops:
        for name, st0 in (("warm_mixed", warm_states), ("prior_mixed", prior_states), ("cold_mixed", None)):
            w = run_steady_batch(ev, states=st0, istop=istop, precision=abi.PREC_MIXED, device=device, rstop=rs)
            dw = dmax(w["states"])
            out[f"{name}_rstop_{rs:g}"] = dict(summ(w), depth_err_vs_steady_median_m=float(np.median(dw)),
                                                depth_err_vs_steady_max_m=max(dw),
                                                within_1cm=int(sum(x <= 0.01 for x in dw)))
    # the other reading of the depth bar: each start against the FP64 cold run's own
    # result at the same stop test (the plain solver's answer, not the steady state)
    def dvs64(states):
        return [float(np.max(np.abs((a["h"] if isinstance(a, dict) else a[0]) - b["h"])))
                for a, b in zip(states, cold64["states"])]
    out["depth_diff_vs_cold_fp64_same_stop"] = {}
    for name, r in (("warm_mixed", warm_mx), ("prior_mixed", prior_mx), ("cold_mixed", cold_mx)):
        dv = dvs64(r["states"])
        out["depth_diff_vs_cold_fp64_same_stop"][name] = {
            "max_m": max(dv), "median_m": float(np.median(dv)), "within_1cm": int(sum(x <= 0.01 for x in dv))}
    out["within_1cm"] = {"warm_mixed": int(sum(x <= 0.01 for x in dh_warm)),
                         "prior_mixed": int(sum(x <= 0.01 for x in dh_prior)),
                         "cold_fp64": int(sum(x <= 0.01 for x in dh_cold64)), "of": len(ev)}
    plain = []
    for sc in ev[:plain_n]:
        pm = fvt.build_mesh(sc.problem)
        opt = abi.default_options(**{f: getattr(sc.options, f) for f, _ in abi.Options._fields_ if f != "reserved"})
        opt.precision = abi.PREC_FP64
        opt.device = device
        with fvt.Solver(pm, opt, keep=pm) as s1:
            s1.set_state(sc.h0, sc.u0, sc.v0)
            s1.step(1)
            s1.set_state(sc.h0, sc.u0, sc.v0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            st = s1.step(istop)
            torch.cuda.synchronize()
            plain.append({"cells": sc.n_elems, "iters": st["iter"], "converged": bool(st["converged"]),
                          "wall_s": time.perf_counter() - t0, "device_s": s1.last_timing()["step_ms"] / 1e3})
    if plain:
        w_plain = float(np.mean([p["wall_s"] for p in plain]))
        warm_wall = (warm_mx["wall_s"] + infer_ms / 1e3 + tm["host_s"] + feat_s) / len(ev)
        out["plain_fp64_single"] = {"scenarios": len(plain), "wall_s_mean": w_plain,
                                    "iters_mean": float(np.mean([p["iters"] for p in plain])),
                                    "converged": int(sum(p["converged"] for p in plain))}
        out["speedup_per_scenario_vs_plain_fp64_single_cold"] = w_plain / warm_wall
        out["warm_batched_wall_s_per_scenario_incl_network"] = warm_wall
        for rs in warm_rstops:
            for name, extra in (("warm_mixed", infer_ms / 1e3 + tm["host_s"] + feat_s), ("prior_mixed", feat_s),
                                ("cold_mixed", 0.0)):
                r = out[f"{name}_rstop_{rs:g}"]
                ww = (r["wall_s_batch"] + extra) / len(ev)
                r["wall_s_per_scenario_incl_preparation"] = ww
                r["speedup_per_scenario_vs_plain_fp64_single_cold"] = w_plain / ww
            r = out[f"warm_mixed_rstop_{rs:g}"]
            r["wall_s_per_scenario_incl_network"] = r["wall_s_per_scenario_incl_preparation"]
    return out


def main(argv=None):
    import argparse
    import json
    ap = argparse.ArgumentParser(description="train and evaluate the steady-state warm start")
    ap.add_argument("--train-n", type=int, default=4096)
    ap.add_argument("--eval-n", type=int, default=64)
    ap.add_argument("--lo", type=int, default=2000)
    ap.add_argument("--hi", type=int, default=8000)
    ap.add_argument("--gen-batch", type=int, default=512)
    ap.add_argument("--istop", type=int, default=40000)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--cells-per-batch", type=int, default=400_000)
    ap.add_argument("--weights-out", default=None)
    ap.add_argument("--json-out", default=None)
    ap.add_argument("--model", default=None, help="evaluate this trained model (.npz) instead of training")
    ap.add_argument("--plain-n", type=int, default=8)
    ap.add_argument("--warm-rstop", type=float, nargs="*", default=[],
                    help="also run the warm start, the prior alone and the cold start to these residuals")
    a = ap.parse_args(argv)
    from . import build
    build.build()
    if a.model:
        import torch
        torch.cuda.set_device(0)
        net, norm = load_model(a.model)
        res = {"model": a.model, "eval": evaluate(net, norm, a.eval_n, a.lo, a.hi, a.istop, plain_n=a.plain_n,
                                                  warm_rstops=a.warm_rstop)}
        s = json.dumps(res)
        print(s)
        if a.json_out:
            with open(a.json_out, "w") as f:
                f.write(s + "\n")
        return
    res = pipeline(a.train_n, a.eval_n, a.lo, a.hi, a.gen_batch, a.istop, a.epochs, a.cells_per_batch, a.lr,
                   weights_out=a.weights_out, log=lambda m: print(m, flush=True), warm_rstops=a.warm_rstop,
                   plain_n=a.plain_n)
    s = json.dumps(res)
    print(s)
    if a.json_out:
        with open(a.json_out, "w") as f:
            f.write(s + "\n")


if __name__ == "__main__":
    main()
